// host_config.cpp -- canonical text configurations (YM-SU2-CONFIG-V1 and its
// SU(3) analogue YM-SU3-CONFIG-V1): the engine's exchange and checkpoint
// format.  Encoding and decoding follow Lattice4::to_canonical_config /
// from_canonical_config (reference/rust/src/lib.rs:587-694) rule for rule,
// including the order in which failures are reported; the SU(3) form adds
// the reference's SU(3) gate (su3.rs:241-252) per link.  Host code, linear
// in the text; compiled with -ffp-contract=off so the norm and residual
// arithmetic is the reference's.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "../../include/ym_config.h"

namespace {

constexpr double kSerializationTolerance = 2.0e-12;   // lib.rs:20
constexpr int64_t kMaxSu2Links = int64_t(1) << 20;     // lib.rs:21 MAX_REFERENCE_LINKS
constexpr int64_t kMaxSu3Links = int64_t(1) << 18;     // su3_lattice.rs:17
constexpr double kSu3Tolerance = 5.0e-12;              // su3.rs:20

struct Group {
    const char *id;
    int words;           // binary64 words per link
    int64_t max_links;
    int32_t too_large;   // status for a lattice over the cap
};
const Group kSu2{YM_SU2_CONFIG_FORMAT_ID, 4, kMaxSu2Links, YM_ERR_LATTICE_TOO_LARGE};
const Group kSu3{YM_SU3_CONFIG_FORMAT_ID, 18, kMaxSu3Links, YM_ERR_LATTICE_TOO_LARGE};

// Lattice4::new_identity / Su3Lattice4::new_identity shape checks
// (lib.rs:242-263, su3_lattice.rs:85-106), in usize arithmetic.
int32_t link_count_u(const uint64_t e[4], const Group &g, bool lift, int64_t *links) {
    for (int d = 0; d < 4; ++d)
        if (e[d] < 2) return YM_ERR_INVALID_LATTICE_EXTENT;
    uint64_t sites = 1;
    for (int d = 0; d < 4; ++d) {
        if (sites > UINT64_MAX / e[d]) return YM_ERR_LATTICE_SIZE_OVERFLOW;
        sites *= e[d];
    }
    if (sites > UINT64_MAX / 4) return YM_ERR_LATTICE_SIZE_OVERFLOW;
    const uint64_t n = sites * 4;
    if (!lift && n > (uint64_t)g.max_links) return g.too_large;
    if (n > (uint64_t)INT64_MAX) return YM_ERR_LATTICE_SIZE_OVERFLOW;
    *links = (int64_t)n;
    return YM_OK;
}

int32_t link_count(const int64_t e[4], const Group &g, bool lift, int64_t *links) {
    uint64_t u[4];
    for (int d = 0; d < 4; ++d) {
        if (e[d] < 2) return YM_ERR_INVALID_LATTICE_EXTENT;
        u[d] = (uint64_t)e[d];
    }
    return link_count_u(u, g, lift, links);
}

// ---------------------------------------------------------------- checks

// Su2::norm_sq (lib.rs:195-197): squares summed left to right.
double su2_norm_sq(const double *c) {
    double s = 0.0;
    for (int k = 0; k < 4; ++k) s += c[k] * c[k];
    return s;
}

// Su2::from_preserved_unit_components (lib.rs:163-177)
int32_t su2_gate(const double *c) {
    for (int k = 0; k < 4; ++k)
        if (!std::isfinite(c[k])) return YM_ERR_NON_FINITE_SU2_COMPONENT;
    for (int k = 0; k < 4; ++k)
        if (std::fabs(c[k]) > 1.0 + kSerializationTolerance) return YM_ERR_NON_UNIT_SU2;
    const double n = su2_norm_sq(c);
    if (!std::isfinite(n) || std::fabs(n - 1.0) > kSerializationTolerance) return YM_ERR_NON_UNIT_SU2;
    return YM_OK;
}

struct Cx {
    double re, im;
};
Cx cadd(Cx a, Cx b) { return {a.re + b.re, a.im + b.im}; }
Cx csub(Cx a, Cx b) { return {a.re - b.re, a.im - b.im}; }
Cx cmul(Cx a, Cx b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
Cx at(const double *m, int r, int c) { return {m[2 * (3 * r + c)], m[2 * (3 * r + c) + 1]}; }

// Mat3::determinant (su3.rs:175-189), cofactor expansion along row 0.
Cx det3(const Cx m[3][3]) {
    const Cx ei = csub(cmul(m[1][1], m[2][2]), cmul(m[1][2], m[2][1]));
    const Cx di = csub(cmul(m[1][0], m[2][2]), cmul(m[1][2], m[2][0]));
    const Cx dh = csub(cmul(m[1][0], m[2][1]), cmul(m[1][1], m[2][0]));
    return cadd(csub(cmul(m[0][0], ei), cmul(m[0][1], di)), cmul(m[0][2], dh));
}

// Su3::from_checked_matrix (su3.rs:241-252) with Mat3::unitarity_residual and
// determinant_residual (su3.rs:219-229): dense products accumulated from
// zero in k order, entry magnitudes by hypot.
int32_t su3_gate(const double *p) {
    for (int k = 0; k < 18; ++k)
        if (!std::isfinite(p[k])) return YM_ERR_NON_FINITE_MATRIX;
    Cx u[3][3], ud[3][3];
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            u[r][c] = at(p, r, c);
            const Cx t = at(p, c, r);
            ud[r][c] = {t.re, -t.im};
        }
    double res = 0.0;
    for (int side = 0; side < 2; ++side) {
        const Cx(*a)[3] = side == 0 ? ud : u;
        const Cx(*b)[3] = side == 0 ? u : ud;
        double mx = 0.0;
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) {
                Cx v{0.0, 0.0};
                for (int k = 0; k < 3; ++k) v = cadd(v, cmul(a[r][k], b[k][c]));
                const Cx d = csub(v, Cx{r == c ? 1.0 : 0.0, 0.0});
                mx = std::fmax(mx, std::hypot(d.re, d.im));
            }
        res = std::fmax(res, mx);
    }
    if (res > kSu3Tolerance) return YM_ERR_NON_UNITARY_MATRIX;
    const Cx d1 = csub(det3(u), Cx{1.0, 0.0}), d2 = csub(det3(ud), Cx{1.0, 0.0});
    if (std::fmax(std::hypot(d1.re, d1.im), std::hypot(d2.re, d2.im)) > kSu3Tolerance)
        return YM_ERR_DETERMINANT_NOT_ONE;
    return YM_OK;
}

int32_t link_gate(const Group &g, const double *link) { return g.words == 4 ? su2_gate(link) : su3_gate(link); }

// Lattice4::max_link_unit_residual (lib.rs:726-740) > tolerance refuses the
// SU(2) encoding; the SU(3) encoding refuses any link its gate refuses.
int32_t encodable(const Group &g, const double *links, int64_t n) {
    for (int64_t l = 0; l < n; ++l) {
        const double *c = links + l * g.words;
        if (g.words == 4) {
            const double r = std::fabs(su2_norm_sq(c) - 1.0);
            if (!std::isfinite(r) || r > kSerializationTolerance) return YM_ERR_NON_UNIT_SU2;
        } else if (int32_t st = su3_gate(c)) {
            return st;
        }
    }
    return YM_OK;
}

// ---------------------------------------------------------------- encode

std::string header(const Group &g, const int64_t e[4], int64_t links) {
    return std::string(g.id) + "\nextents=" + std::to_string(e[0]) + "," + std::to_string(e[1]) + "," +
           std::to_string(e[2]) + "," + std::to_string(e[3]) + "\nlink_count=" + std::to_string(links) + "\n";
}

void put_hex(char *o, double v) {
    static const char digits[] = "0123456789abcdef";
    uint64_t b;
    std::memcpy(&b, &v, 8);
    for (int k = 15; k >= 0; --k) {
        o[k] = digits[b & 15];
        b >>= 4;
    }
}

int32_t encode(const Group &g, const int64_t *e, const double *links, int32_t lift, char *text,
               int64_t capacity, int64_t *length) {
    if (!e || !links || !length) return YM_ERR_NULL_ARGUMENT;
    int64_t n = 0;
    if (int32_t st = link_count(e, g, lift != 0, &n)) return st;
    if (int32_t st = encodable(g, links, n)) return st;
    const std::string h = header(g, e, n);
    const int64_t line = 17 * g.words;   // words of 16 digits, separators and the newline
    if (n > (INT64_MAX - (int64_t)h.size()) / line) return YM_ERR_LATTICE_SIZE_OVERFLOW;
    const int64_t total = (int64_t)h.size() + n * line;
    *length = total;
    if (!text) return YM_OK;
    if (capacity < total) return YM_ERR_SCRATCH_TOO_SMALL;
    std::memcpy(text, h.data(), h.size());
    char *o = text + h.size();
    for (int64_t l = 0; l < n; ++l) {
        for (int k = 0; k < g.words; ++k) {
            put_hex(o, links[l * g.words + k]);
            o[16] = k + 1 == g.words ? '\n' : ',';
            o += 17;
        }
    }
    return YM_OK;
}

// ---------------------------------------------------------------- decode

// str::lines(): split at "\n" or "\r\n"; the final line ending is optional.
// `canonical` is cleared by any "\r\n" ending or a missing final newline,
// which the reference's closing comparison with the re-encoding rejects.
struct Lines {
    const char *p, *end;
    bool canonical = true;
    bool next(const char **b, int64_t *n) {
        if (p >= end) return false;
        const char *nl = (const char *)std::memchr(p, '\n', (size_t)(end - p));
        const char *stop = nl ? nl : end;
        const char *line_end = stop;
        if (nl && line_end > p && line_end[-1] == '\r') {
            --line_end;
            canonical = false;
        }
        if (!nl) canonical = false;
        *b = p;
        *n = line_end - p;
        p = nl ? nl + 1 : end;
        return true;
    }
};

bool starts_with(const char *b, int64_t n, const char *prefix, int64_t *skip) {
    const int64_t k = (int64_t)std::strlen(prefix);
    if (n < k || std::memcmp(b, prefix, (size_t)k) != 0) return false;
    *skip = k;
    return true;
}

// <usize as FromStr>: an optional '+', then one or more ASCII digits, no
// overflow.  `canonical` is cleared by a '+' or a redundant leading zero.
bool parse_usize(const char *b, int64_t n, uint64_t *out, bool *canonical) {
    if (n > 0 && b[0] == '+') {
        ++b;
        --n;
        *canonical = false;
    }
    if (n == 0) return false;
    if (n > 1 && b[0] == '0') *canonical = false;
    uint64_t v = 0;
    for (int64_t i = 0; i < n; ++i) {
        if (b[i] < '0' || b[i] > '9') return false;
        const uint64_t d = (uint64_t)(b[i] - '0');
        if (v > (UINT64_MAX - d) / 10) return false;
        v = v * 10 + d;
    }
    *out = v;
    return true;
}

bool hex16(const char *b, uint64_t *out) {
    uint64_t v = 0;
    for (int i = 0; i < 16; ++i) {
        const char ch = b[i];
        uint64_t d;
        if (ch >= '0' && ch <= '9') d = (uint64_t)(ch - '0');
        else if (ch >= 'a' && ch <= 'f') d = (uint64_t)(ch - 'a' + 10);
        else return false;
        v = (v << 4) | d;
    }
    *out = v;
    return true;
}

int32_t decode(const Group &g, const char *text, int64_t length, int32_t lift, int64_t *e_out,
               double *links, int64_t capacity) {
    constexpr int32_t kBad = YM_ERR_INVALID_CONFIGURATION_ENCODING;
    if (!text || !e_out) return YM_ERR_NULL_ARGUMENT;
    Lines lines{text, text + (length > 0 ? length : 0)};
    const char *b;
    int64_t n, skip;
    bool canonical = true;
    if (!lines.next(&b, &n) || n != (int64_t)std::strlen(g.id) || std::memcmp(b, g.id, (size_t)n) != 0)
        return kBad;
    if (!lines.next(&b, &n) || !starts_with(b, n, "extents=", &skip)) return kBad;
    uint64_t ext[4];
    {
        const char *q = b + skip, *qend = b + n;
        for (int d = 0; d < 4; ++d) {
            if (q > qend) return kBad;   // fewer than four parts
            const char *comma = (const char *)std::memchr(q, ',', (size_t)(qend - q));
            const char *stop = comma ? comma : qend;
            if (!parse_usize(q, stop - q, &ext[d], &canonical)) return kBad;
            q = comma ? comma + 1 : qend + 1;
        }
        if (q <= qend) return kBad;   // a fifth part
    }
    if (!lines.next(&b, &n) || !starts_with(b, n, "link_count=", &skip)) return kBad;
    uint64_t declared;
    if (!parse_usize(b + skip, n - skip, &declared, &canonical)) return kBad;
    if (!lift && declared > (uint64_t)g.max_links) return g.too_large;
    int64_t count = 0;
    if (int32_t st = link_count_u(ext, g, lift != 0, &count)) return st;
    if (declared != (uint64_t)count) return kBad;
    for (int d = 0; d < 4; ++d) e_out[d] = (int64_t)ext[d];
    if (!links) return YM_OK;
    if (capacity < count) return YM_ERR_SCRATCH_TOO_SMALL;
    double w[18];
    for (int64_t l = 0; l < count; ++l) {
        if (!lines.next(&b, &n)) return kBad;
        const char *q = b, *qend = b + n;
        for (int k = 0; k < g.words; ++k) {
            if (q > qend) return kBad;
            const char *comma = (const char *)std::memchr(q, ',', (size_t)(qend - q));
            const char *stop = comma ? comma : qend;
            uint64_t bits;
            if (stop - q != 16 || !hex16(q, &bits)) return kBad;
            std::memcpy(&w[k], &bits, 8);
            q = comma ? comma + 1 : qend + 1;
        }
        if (q <= qend) return kBad;
        if (int32_t st = link_gate(g, w)) return st;
        std::memcpy(links + l * g.words, w, sizeof(double) * (size_t)g.words);
    }
    if (lines.next(&b, &n)) return kBad;
    if (!canonical || !lines.canonical) return kBad;   // not the canonical re-encoding
    return YM_OK;
}

}  // namespace

extern "C" {

int32_t ym_su2_to_canonical_config(const int64_t extents[4], const double *links,
                                   int32_t lift_reference_caps, char *text, int64_t capacity,
                                   int64_t *length) {
    return encode(kSu2, extents, links, lift_reference_caps, text, capacity, length);
}

int32_t ym_su2_from_canonical_config(const char *text, int64_t length, int32_t lift_reference_caps,
                                     int64_t extents[4], double *links, int64_t links_capacity) {
    return decode(kSu2, text, length, lift_reference_caps, extents, links, links_capacity);
}

int32_t ym_su3_to_canonical_config(const int64_t extents[4], const double *links,
                                   int32_t lift_reference_caps, char *text, int64_t capacity,
                                   int64_t *length) {
    return encode(kSu3, extents, links, lift_reference_caps, text, capacity, length);
}

int32_t ym_su3_from_canonical_config(const char *text, int64_t length, int32_t lift_reference_caps,
                                     int64_t extents[4], double *links, int64_t links_capacity) {
    return decode(kSu3, text, length, lift_reference_caps, extents, links, links_capacity);
}

}  // extern "C"

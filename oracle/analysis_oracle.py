"""Pure-Python restatement of the reference's glueball correlator analysis.

TEST INFRASTRUCTURE ONLY.  Restates, in plain Python floats (IEEE binary64,
no contraction), the reference crate's (QSOLKCB/YANG-MILLS,
``reference/rust/src``) periodic cosh effective mass
(``glueball_effective_mass.rs``), correlated single-state fit
(``glueball_scalar_fit.rs``) and two-operator variational projection
(``glueball_scalar_variational.rs``).  The test-suite checks the engine's
host analysis (``include/ym_analysis.h``) against it bit for bit and pins it
to the reference's golden vectors; the product never imports it.

Transcendentals are the platform libm the reference links (``exp``, ``log``,
``hypot`` through ctypes, so ``hypot`` is glibc's and not CPython's own);
Rust's ``f64::acosh`` is ``ln(x + sqrt(x - 1) sqrt(x + 1))``; ``f64::mul_add``
is an exactly rounded fused multiply-add, computed here with fractions.
Errors are raised as ``AnalysisError(variant)`` with the reference's
variant names.  Sized for small cases (pure-Python loops).
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
from fractions import Fraction

_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.hypot.argtypes = [ctypes.c_double, ctypes.c_double]
_libm.hypot.restype = ctypes.c_double
_libm.exp.argtypes = [ctypes.c_double]
_libm.exp.restype = ctypes.c_double
_libm.log.argtypes = [ctypes.c_double]
_libm.log.restype = ctypes.c_double


class AnalysisError(ValueError):
    def __init__(self, variant: str):
        super().__init__(variant)
        self.variant = variant


def _fin(x: float) -> bool:
    return math.isfinite(x)


def hypot(a: float, b: float) -> float:
    return _libm.hypot(a, b)


def exp(x: float) -> float:
    return _libm.exp(x)


def fma(a: float, b: float, c: float) -> float:
    """Exactly rounded a*b + c (f64::mul_add)."""
    if not (_fin(a) and _fin(b) and _fin(c)):
        return a * b + c
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def rust_acosh(x: float) -> float:
    if x < 1.0:
        return math.nan
    return _libm.log(x + math.sqrt(x - 1.0) * math.sqrt(x + 1.0))


def rust_max(a: float, b: float) -> float:
    """f64::max: the non-NaN operand wins."""
    if math.isnan(a):
        return b
    if math.isnan(b):
        return a
    return a if a >= b else b


# ---------------------------------------------------------------- phase 3D

def _validate_effective_mass(full, jackknife, lags):   # glueball_effective_mass.rs:91-134
    nt = len(full)
    if nt < 4:
        raise AnalysisError("TimeExtentTooSmall")
    if nt > 64:
        raise AnalysisError("TimeExtentTooLarge")
    if len(jackknife) < 3:
        raise AnalysisError("TooFewJackknifeReplicates")
    if len(jackknife) > 64:
        raise AnalysisError("TooManyJackknifeReplicates")
    if not lags:
        raise AnalysisError("EmptyAnalysisWindow")
    if any(not _fin(v) for v in full):
        raise AnalysisError("NonFiniteCorrelator")
    if any(len(r) != nt for r in jackknife):
        raise AnalysisError("ShapeMismatch")
    if any(not _fin(v) for r in jackknife for v in r):
        raise AnalysisError("NonFiniteCorrelator")
    prev = 0
    for i, tau in enumerate(lags):
        if tau == 0 or tau >= nt - 1 or 2 * tau >= nt or (i != 0 and tau <= prev):
            raise AnalysisError("InvalidAnalysisLag")
        prev = tau


def _cosh_mass(c, tau):   # glueball_effective_mass.rs:136-157
    center = c[tau]
    if center <= 0.0:
        raise AnalysisError("NonPositiveCentralCorrelator")
    num = c[tau - 1] + c[tau + 1]
    den = 2.0 * center
    if not (_fin(num) and _fin(den)):
        raise AnalysisError("NonFiniteStatistic")
    arg = num / den
    if not _fin(arg):
        raise AnalysisError("NonFiniteStatistic")
    if arg < 1.0:
        raise AnalysisError("AcoshDomainViolation")
    m = rust_acosh(arg)
    if not _fin(m):
        raise AnalysisError("NonFiniteStatistic")
    return m


def cosh_effective_mass_with_jackknife(full, jackknife, lags):
    """glueball_effective_mass.rs:170-234 -> [(tau, full, mean, se)]."""
    full = [float(v) for v in full]
    jackknife = [[float(v) for v in r] for r in jackknife]
    lags = [int(t) for t in lags]
    _validate_effective_mass(full, jackknife, lags)
    out = []
    for tau in lags:
        est = _cosh_mass(full, tau)
        ms, s = [], 0.0
        for r in jackknife:
            m = _cosh_mass(r, tau)
            s += m
            if not _fin(s):
                raise AnalysisError("NonFiniteStatistic")
            ms.append(m)
        n = float(len(ms))
        mean = s / n
        ssd = 0.0
        for m in ms:
            d = m - mean
            ssd += d * d
        var = ((n - 1.0) / n) * ssd
        se = math.sqrt(var)
        out.append((tau, est, mean, se))
    return out


def analytic_periodic_single_state(nt, mass, amplitude):   # glueball_effective_mass.rs:237-263
    if not (4 <= nt <= 64) or not _fin(mass) or mass <= 0.0 or not _fin(amplitude) or amplitude <= 0.0:
        raise AnalysisError("InvalidFixtureParameter")
    return [amplitude * (exp(-mass * float(t)) + exp(-mass * float(nt - t))) for t in range(nt)]


# ---------------------------------------------------------------- phase 3E

def _count(w):
    s, e = w
    return e - s + 1 if e >= s else None


def _validate_windows(nt, cands):   # glueball_scalar_fit.rs:156-182
    if not cands:
        raise AnalysisError("EmptyCandidateWindows")
    if len(cands) > 16:
        raise AnalysisError("TooManyCandidateWindows")
    for i, w in enumerate(cands):
        c = _count(w)
        if c is None or w[0] == 0 or c < 3 or c > 8 or 2 * w[1] >= nt:
            raise AnalysisError("InvalidCandidateWindow")
        if w in cands[:i]:
            raise AnalysisError("DuplicateCandidateWindow")


def _plateau(full, jk, w):   # glueball_scalar_fit.rs:197-237
    pts = cosh_effective_mass_with_jackknife(full, jk, list(range(w[0], w[1] + 1)))
    ws = wt = 0.0
    for _, est, _, se in pts:
        if not _fin(se) or se <= 0.0:
            raise AnalysisError("DegeneratePlateauUncertainty")
        weight = 1.0 / (se * se)
        ws += weight * est
        wt += weight
    wm = ws / wt
    mz = 0.0
    for _, est, _, se in pts:
        mz = rust_max(mz, abs((est - wm) / se))
    return wm, mz


def choose_plateau_window(full, jk, cands):   # glueball_scalar_fit.rs:239-274
    _validate_windows(len(full), cands)
    best = None
    for w in cands:
        try:
            wm, mz = _plateau(full, jk, w)
        except AnalysisError as e:
            if e.variant == "DegeneratePlateauUncertainty":
                continue
            raise
        if mz > 2.5:
            continue
        if best is None or _count(w) > _count(best[0]) or (_count(w) == _count(best[0]) and w[0] > best[0][0]):
            best = (w, wm, mz)
    if best is None:
        raise AnalysisError("NoAcceptedPlateauWindow")
    return best


def jackknife_covariance(jk, w):   # glueball_scalar_fit.rs:276-322
    p = _count(w)
    if len(jk) <= p:
        raise AnalysisError("InsufficientReplicatesForCovariance")
    means = [0.0] * p
    for r in jk:
        for c in range(p):
            means[c] += r[w[0] + c]
    n = float(len(jk))
    means = [m / n for m in means]
    cov = [[0.0] * p for _ in range(p)]
    for r in jk:
        for a in range(p):
            left = r[w[0] + a] - means[a]
            for b in range(p):
                cov[a][b] += left * (r[w[0] + b] - means[b])
    f = (n - 1.0) / n
    return [[x * f for x in row] for row in cov]


def _check_pd(m):   # glueball_scalar_fit.rs:324-359
    n = len(m)
    scale = 0.0
    for row in m:
        for x in row:
            scale = rust_max(scale, abs(x))
    if not _fin(scale) or scale <= 0.0:
        raise AnalysisError("CovarianceNotPositiveDefinite")
    low = [[0.0] * n for _ in range(n)]
    for i in range(n):
        for j in range(i + 1):
            s = m[i][j]
            for k in range(j):
                s -= low[i][k] * low[j][k]
            if i == j:
                if not _fin(s) or s <= scale * 1.0e-12:
                    raise AnalysisError("CovarianceNotPositiveDefinite")
                low[i][j] = math.sqrt(s)
            else:
                low[i][j] = s / low[j][j]
    return scale


def invert_matrix(m):   # glueball_scalar_fit.rs:361-421
    m = [[float(x) for x in row] for row in m]
    scale = _check_pd(m)
    n = len(m)
    aug = [row[:] + [1.0 if c == r else 0.0 for c in range(n)] for r, row in enumerate(m)]
    for col in range(n):
        pr, pa = col, abs(aug[col][col])
        for r in range(col + 1, n):
            if abs(aug[r][col]) > pa:
                pa, pr = abs(aug[r][col]), r
        if not _fin(pa) or pa <= scale * 1.0e-12:
            raise AnalysisError("SingularCovariance")
        aug[col], aug[pr] = aug[pr], aug[col]
        piv = aug[col][col]
        aug[col] = [x / piv for x in aug[col]]
        for r in range(n):
            if r == col:
                continue
            f = aug[r][col]
            aug[r] = [x - f * y for x, y in zip(aug[r], aug[col])]
    return [row[n:] for row in aug]


def _quad(left, m, right):   # glueball_scalar_fit.rs:423-439
    s = 0.0
    for i in range(len(m)):
        inner = 0.0
        for c in range(len(m)):
            inner += m[i][c] * right[c]
        s += left[i] * inner
    if not _fin(s):
        raise AnalysisError("NonFiniteStatistic")
    return s


def profile_grid_fit(nt, w, values, inv):   # glueball_scalar_fit.rs:470-526
    best = None
    for g in range(1951):
        mass = 0.05 + 0.001 * float(g)
        if mass > 2.0 + 1.0e-15:
            break
        basis = [exp(-mass * float(t)) + exp(-mass * float(nt - t)) for t in range(w[0], w[1] + 1)]
        den = _quad(basis, inv, basis)
        if den <= 0.0:
            continue
        amp = _quad(basis, inv, values) / den
        if amp <= 0.0 or not _fin(amp):
            continue
        res = [v - amp * b for v, b in zip(values, basis)]
        chi2 = _quad(res, inv, res)
        if chi2 < 0.0:
            continue
        if best is None or chi2 < best[2] or (chi2 == best[2] and mass < best[0]):
            best = (mass, amp, chi2)
    if best is None:
        raise AnalysisError("NoFiniteGridFit")
    return best


def _jk_error(v):   # glueball_scalar_fit.rs:548-565
    n = float(len(v))
    s = 0.0
    for x in v:
        s += x
    mean = s / n
    ssd = 0.0
    for x in v:
        ssd += (x - mean) * (x - mean)
    return mean, math.sqrt(((n - 1.0) / n) * ssd)


def maximum_off_diagonal_correlation(cov):   # glueball_scalar_fit.rs:567-593
    mx = 0.0
    for r in range(len(cov)):
        if cov[r][r] <= 0.0:
            raise AnalysisError("CovarianceNotPositiveDefinite")
        rs = math.sqrt(cov[r][r])
        for c in range(r):
            if cov[c][c] <= 0.0:
                raise AnalysisError("CovarianceNotPositiveDefinite")
            mx = rust_max(mx, abs((cov[r][c] / rs) / math.sqrt(cov[c][c])))
    return mx


def correlated_scalar_fit(full, jk, cands):
    """glueball_scalar_fit.rs:595-650 -> dict of the ScalarFitResult fields."""
    full = [float(v) for v in full]
    jk = [[float(v) for v in r] for r in jk]
    cands = [tuple(int(x) for x in w) for w in cands]
    w, wm, mz = choose_plateau_window(full, jk, cands)
    cov = jackknife_covariance(jk, w)
    inv = invert_matrix(cov)
    corr = maximum_off_diagonal_correlation(cov)
    sl = slice(w[0], w[1] + 1)
    fm, fa, fc = profile_grid_fit(len(full), w, full[sl], inv)
    fits = [profile_grid_fit(len(full), w, r[sl], inv) for r in jk]
    mm, mse = _jk_error([f[0] for f in fits])
    am, ase = _jk_error([f[1] for f in fits])
    dof = _count(w) - 2
    return dict(time_extent=len(full), jackknife_replicates=len(jk), selected_window=w,
                plateau_weighted_effective_mass=wm, plateau_maximum_z=mz, fitted_mass=fm,
                fitted_amplitude=fa, chi_square=fc, degrees_of_freedom=dof,
                chi_square_per_dof=fc / float(dof), mass_jackknife_mean=mm, mass_standard_error=mse,
                amplitude_jackknife_mean=am, amplitude_standard_error=ase,
                maximum_off_diagonal_correlation=corr)


# ---------------------------------------------------------------- phase 3J

def _stable_average(x, y):   # glueball_scalar_variational.rs:149-165
    if x == y and math.copysign(1.0, x) == math.copysign(1.0, y):
        return x
    return x + 0.5 * (y - x)


def _sym(m):
    c = _stable_average(m[0][1], m[1][0])
    return [[m[0][0], c], [c, m[1][1]]]


def _validate_series(mats):   # glueball_scalar_variational.rs:132-185
    if len(mats) < 3 or len(mats) > 64:
        raise AnalysisError("CorrelatorShapeMismatch")
    for m in mats:
        if not all(_fin(x) for row in m for x in row):
            raise AnalysisError("NonFiniteAccumulator")
        res = abs(m[0][1] - m[1][0])
        scale = rust_max(rust_max(abs(m[0][1]), abs(m[1][0])), 1.0)
        if not _fin(res) or res > 2.0e-12 * scale:
            raise AnalysisError("MatrixNotSymmetric")


def _divide_by_product(num, p, q):   # glueball_scalar_variational.rs:207-248
    if p == 0.0 or q == 0.0:
        raise AnalysisError("NonFiniteAccumulator")
    large, small = (p, q) if abs(p) >= abs(q) else (q, p)
    i1 = num / large
    v1 = i1 / small
    if _fin(i1) and _fin(v1) and (i1 != 0.0 or num == 0.0):
        return v1
    i2 = num / small
    v2 = i2 / large
    if _fin(i2) and _fin(v2):
        return v2
    raise AnalysisError("NonFiniteAccumulator")


def _compensated_det(a, d, c):   # glueball_scalar_variational.rs:250-282
    ad, cc = a * d, c * c
    return (ad - cc) + (fma(a, d, -ad) - fma(c, c, -cc))


def _characteristic_root(rdet, roff, d1, d2, off):   # glueball_scalar_variational.rs:284-378
    if not (_fin(d1) and _fin(d2) and _fin(off)):
        raise AnalysisError("NonFiniteAccumulator")
    pd, md, sd = 1.0 + roff, 1.0 - roff, math.sqrt(rdet)
    if pd <= 0.0 or md <= 0.0 or sd <= 0.0:
        raise AnalysisError("ReferenceMatrixNotPositiveDefinite")
    avg = 0.5 * d1 + 0.5 * d2
    plus, minus, cross = avg + off, avg - off, 0.5 * d1 - 0.5 * d2
    if not all(_fin(x) for x in (avg, plus, minus, cross)):
        raise AnalysisError("NonFiniteAccumulator")
    t1, t2, toff = plus / pd, minus / md, cross / sd
    if not all(_fin(x) for x in (t1, t2, toff)):
        raise AnalysisError("NonFiniteAccumulator")
    if toff == 0.0 and t1 == t2:
        raise AnalysisError("DegeneratePrincipalEigenvector")
    mid, half = 0.5 * t1 + 0.5 * t2, 0.5 * t1 - 0.5 * t2
    radius = hypot(half, toff)
    if not (_fin(mid) and _fin(half) and _fin(radius)):
        raise AnalysisError("NonFiniteAccumulator")
    if radius == 0.0:
        raise AnalysisError("DegeneratePrincipalEigenvector")
    if mid >= 0.0:
        root = mid + radius
        if not _fin(root):
            raise AnalysisError("NonFiniteAccumulator")
        return root
    smaller = mid - radius
    if not _fin(smaller) or smaller == 0.0:
        raise AnalysisError("NonFiniteAccumulator")
    return _divide_by_product(_compensated_det(d1, d2, off), rdet, smaller)


def principal_eigenvalue(c0, c1):   # glueball_scalar_variational.rs:380-464
    r, g = _sym(c0), _sym(c1)
    r1, r2 = r[0][0], r[1][1]
    if r1 <= 0.0 or r2 <= 0.0:
        raise AnalysisError("ReferenceMatrixNotPositiveDefinite")
    rs = math.sqrt(r1) * math.sqrt(r2)
    roff = r[0][1] / rs
    rdet = 1.0 - roff * roff
    if not _fin(roff) or rdet <= 1.0e-14:
        raise AnalysisError("ReferenceMatrixNotPositiveDefinite")
    d1, d2, off = g[0][0] / r1, g[1][1] / r2, g[0][1] / rs
    if roff == 0.0 and off == 0.0:
        if d1 == d2:
            raise AnalysisError("DegeneratePrincipalEigenvector")
        return rust_max(d1, d2)
    try:
        return _characteristic_root(rdet, roff, d1, d2, off)
    except AnalysisError as e:
        if e.variant != "NonFiniteAccumulator":
            raise
    scale = rust_max(rust_max(abs(d1), abs(d2)), abs(off))
    if not _fin(scale) or scale <= 0.0:
        raise AnalysisError("NonFiniteAccumulator")
    root = scale * _characteristic_root(rdet, roff, d1 / scale, d2 / scale, off / scale)
    if not _fin(root):
        raise AnalysisError("NonFiniteAccumulator")
    return root


def _whiten(m, first, second, dscale, roff, rdet):   # glueball_scalar_variational.rs:481-566
    m = _sym(m)
    n1, n2, no = m[0][0] / first, m[1][1] / second, m[0][1] / dscale
    if not (_fin(n1) and _fin(n2) and _fin(no)):
        raise AnalysisError("NonFiniteAccumulator")
    if roff == 0.0:
        return [[n1, no], [no, n2]]
    scale = rust_max(rust_max(abs(n1), abs(n2)), abs(no))
    if scale == 0.0:
        return [[0.0, 0.0], [0.0, 0.0]]
    f, s, o = n1 / scale, n2 / scale, no / scale
    sd = math.sqrt(rdet)
    w12 = fma(-roff, f, o) / sd
    w22 = fma(roff, roff * f, fma(-2.0 * roff, o, s)) / rdet
    out = [[f * scale, w12 * scale], [w12 * scale, w22 * scale]]
    if not all(_fin(x) for row in out for x in row):
        raise AnalysisError("NonFiniteAccumulator")
    return out


def principal_generalized_projection(mats, t0=1, t1=2):
    """glueball_scalar_variational.rs:746-925 -> (lambda, (c0, c1), projected)."""
    mats = [[[float(x) for x in row] for row in m] for m in mats]
    _validate_series(mats)
    if t0 != 1 or t1 != 2 or t1 >= len(mats):
        raise AnalysisError("InvalidReferenceTimes")
    c0, c1 = _sym(mats[t0]), _sym(mats[t1])
    a, d = c0[0][0], c0[1][1]
    if a <= 0.0 or d <= 0.0:
        raise AnalysisError("ReferenceMatrixNotPositiveDefinite")
    ds = math.sqrt(a) * math.sqrt(d)
    noff = c0[0][1] / ds
    ndet = 1.0 - noff * noff
    if not _fin(noff) or ndet <= 1.0e-14:
        raise AnalysisError("ReferenceMatrixNotPositiveDefinite")
    l00, l10 = math.sqrt(a), c0[1][0] / math.sqrt(a)
    l11 = math.sqrt(d) * math.sqrt(ndet)
    q = _divide_by_product(l10, l00, l11)
    w = _whiten(c1, a, d, ds, noff, ndet)
    lam = principal_eigenvalue(c0, c1)
    if lam <= 0.0:
        raise AnalysisError("NonPositivePrincipalEigenvalue")
    wa, wd, wo = w[0][0], w[1][1], w[0][1]
    if wo != 0.0:
        half = 0.5 * wa - 0.5 * wd
        rad = hypot(half, wo)
        if rad == 0.0:
            raise AnalysisError("DegeneratePrincipalEigenvector")
        cs = rust_max(rust_max(abs(rad), abs(half)), abs(wo))
        e = [rad / cs + half / cs, wo / cs] if half >= 0.0 else [wo / cs, rad / cs - half / cs]
    elif wa > wd:
        e = [1.0, 0.0]
    elif wd > wa:
        e = [0.0, 1.0]
    else:
        raise AnalysisError("DegeneratePrincipalEigenvector")
    en = hypot(e[0], e[1])
    e = [e[0] / en, e[1] / en]
    inv00, inv10, inv11 = 1.0 / l00, -q, 1.0 / l11
    c = [inv00 * e[0] + inv10 * e[1], 0.0 * e[0] + inv11 * e[1]]
    first, second = l00 * c[0] + l10 * c[1], l11 * c[1]
    norm = hypot(first, second)
    if not _fin(norm) or norm <= 0.0:
        raise AnalysisError("ProjectionNormalizationFailure")
    c = [c[0] / norm, c[1] / norm]
    if abs(c[0]) > 1.0e-14:
        if c[0] < 0.0:
            c = [-c[0], -c[1]]
    elif c[1] < 0.0:
        c = [-c[0], -c[1]]
    mv = [l00 * c[0] + l10 * c[1], l11 * c[1]]
    mn = hypot(mv[0], mv[1])
    if abs(mn * mn - 1.0) > 2.0e-12:
        raise AnalysisError("ProjectionNormalizationFailure")
    proj = []
    for t, m in enumerate(mats):
        if t == t0:
            proj.append(1.0)
        elif t == t1:
            proj.append(lam)
        else:
            ms = _sym(m)
            if ms == c0:
                proj.append(1.0)
                continue
            wm = _whiten(ms, a, d, ds, noff, ndet)
            r0 = fma(wm[0][0], mv[0], wm[0][1] * mv[1])
            r1 = fma(wm[1][0], mv[0], wm[1][1] * mv[1])
            proj.append(fma(mv[0], r0, mv[1] * r1))
    return lam, (c[0], c[1]), proj


def variational_correlator_from_samples(plaq, rect):
    """glueball_scalar_variational.rs:628-744 from samples[cfg][t]."""
    ncfg, nt = len(plaq), len(plaq[0])
    if ncfg == 0:
        raise AnalysisError("EmptyConfigurationSet")
    if ncfg > 64:
        raise AnalysisError("TooManyConfigurations")
    if nt < 3:
        raise AnalysisError("TimeExtentTooSmall")
    if nt > 64:
        raise AnalysisError("TimeExtentTooLarge")
    s0 = s1 = 0.0
    for c in range(ncfg):
        for t in range(nt):
            s0 += plaq[c][t]
            s1 += rect[c][t]
    norm = float(ncfg * nt)
    v0, v1 = s0 / norm, s1 / norm
    mats = []
    for tau in range(nt):
        pp = rr = pr = rp = 0.0
        for c in range(ncfg):
            for t in range(nt):
                u = (t + tau) % nt
                pp += plaq[c][t] * plaq[c][u]
                rr += rect[c][t] * rect[c][u]
                pr += plaq[c][t] * rect[c][u]
                rp += rect[c][t] * plaq[c][u]
        cross = 0.5 * (pr / norm + rp / norm) - v0 * v1
        mats.append([[pp / norm - v0 * v0, cross], [cross, rr / norm - v1 * v1]])
    return (v0, v1), mats

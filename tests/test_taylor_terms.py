"""Term counts of the fixed-length rotation chains of the FP64 sub-sweep.

The ordered-hit sub-sweep evaluates each hit's rotation entries with a
fixed number K of the reference's Taylor terms (csrc/su3_tiled.cuh
taylor_fixed / lambda8_fixed: t_k = (t_{k-1} h) fl(1/k), added to the
cosine or sine sum unless an earlier term was at or below the reference's
1e-18 cutoff, su3.rs:25,434-440).  Every term past the cutoff the reference
would still add has to be either skipped by that rule or too small to move
the sum (below half an ulp of it), or the kernel's bits would differ from
the reference's.  For half widths a <= 0.3 the kernel takes K = 11: the
terms t_12 <= 0.1732^12/12! = 1.5e-18 and t_13 <= 2e-20 are far below half
an ulp of sums near cos h ~ 0.985 (5.6e-17) and sin h ~ h.  For a <= 1 it
takes K = 14: t_15 / s <= 0.5^14/15! = 4.7e-17 stays below the smallest
relative half ulp, 2^-54 = 5.55e-17.  So K and the reference's open-ended
loop give the same c and s.

The chains are replayed here in binary64 with numpy (each product and sum
rounded once, as in the kernel, which is compiled without fused
multiply-adds) over random grid angles and the grid's extremes, and K = 11
(K = 14) is checked bitwise against the loop run to the cutoff, and one
term fewer is shown to differ.
"""
import numpy as np

INV = np.array([0.0] + [1.0 / k for k in range(1, 68)])
CUTOFF = 1.0e-18
INV_SQRT3 = 0.5773502691896258


def _grid_thetas(a, n, seed):
    """Angles of the paired grid (proposal_angle_from_u64, su3_ensemble.rs:199-213)."""
    rng = np.random.default_rng(seed)
    m = rng.integers(0, 1 << 52, size=n, dtype=np.uint64)
    m = np.concatenate([m, np.array([0, 1, (1 << 52) - 1, (1 << 52) - 2], np.uint64)])
    sign = np.where(rng.integers(0, 2, size=m.size) == 0, -1.0, 1.0)
    sign[-4:] = [1.0, -1.0, 1.0, -1.0]
    mag = a * (2.0 * m.astype(np.float64) + 1.0) * (1.0 / 9007199254740992.0)
    return sign * mag


def _chains(hs, K):
    """Lockstep chains of the cosine/sine sums; one shared stop flag on the
    largest term (for a single chain: that chain's term)."""
    t = [np.ones_like(h) for h in hs]
    c = [np.ones_like(h) for h in hs]
    s = [np.zeros_like(h) for h in hs]
    done = np.zeros(hs[0].shape, bool)
    for k in range(1, K + 1):
        big = np.zeros_like(hs[0])
        for i, h in enumerate(hs):
            t[i] = (t[i] * h) * INV[k]
            if k % 4 == 1:
                s[i] = np.where(done, s[i], s[i] + t[i])
            elif k % 4 == 2:
                c[i] = np.where(done, c[i], c[i] - t[i])
            elif k % 4 == 3:
                s[i] = np.where(done, s[i], s[i] - t[i])
            else:
                c[i] = np.where(done, c[i], c[i] + t[i])
            big = np.maximum(big, np.abs(t[i]))
        done = done | (big <= CUTOFF)
    return c, s, done


def test_block_rotation_needs_eleven_terms_at_half_width_03():
    h = 0.5 * _grid_thetas(0.3, 2_000_000, 1)
    c11, s11, _ = _chains([h], 11)
    c13, s13, _ = _chains([h], 13)
    c64, s64, done = _chains([h], 64)
    assert done.all()                       # the reference's loop stops within 64 terms
    for a, b in ((c11, c13), (s11, s13), (c11, c64), (s11, s64)):
        assert np.array_equal(a[0], b[0])
    c10, s10, _ = _chains([h], 10)          # and eleven are needed
    assert not np.array_equal(s10[0], s11[0])


def test_lambda8_rotation_needs_eleven_terms_at_half_width_03():
    theta = _grid_thetas(0.3, 2_000_000, 2)
    d1, d2 = (0.5 * INV_SQRT3) * theta, (-INV_SQRT3) * theta
    assert max(np.abs(d1).max(), np.abs(d2).max()) <= 0.5   # no halving and squaring
    r11 = _chains([d1, d2], 11)
    r13 = _chains([d1, d2], 13)
    r64 = _chains([d1, d2], 64)
    assert r64[2].all()
    for i in range(2):
        for part in (0, 1):
            assert np.array_equal(r11[part][i], r13[part][i])
            assert np.array_equal(r11[part][i], r64[part][i])


def test_rotations_need_fourteen_terms_at_half_width_1():
    h = 0.5 * _grid_thetas(1.0, 1_000_000, 3)
    ref = _chains([h], 64)
    assert ref[2].all()
    r14, r13 = _chains([h], 14), _chains([h], 13)
    assert all(np.array_equal(r14[p][0], ref[p][0]) for p in (0, 1))
    assert not all(np.array_equal(r13[p][0], ref[p][0]) for p in (0, 1))
    # lambda8: one halving (and a squaring afterwards) once |theta|/sqrt(3) > 1/2
    theta = _grid_thetas(1.0, 1_000_000, 4)
    d1, d2 = (0.5 * INV_SQRT3) * theta, (-INV_SQRT3) * theta
    sc = np.where(np.maximum(np.abs(d1), np.abs(d2)) > 0.5, 0.5, 1.0)
    h1, h2 = d1 * sc, d2 * sc
    ref = _chains([h1, h2], 64)
    r14 = _chains([h1, h2], 14)
    assert all(np.array_equal(r14[p][i], ref[p][i]) for p in (0, 1) for i in (0, 1))

"""The oracle of the learned proposal checked against first principles: the
closed-form ReTr(R_a(theta) M) against the exact rotation matrices, the
analytic objective gradient against finite differences, gauge invariance
of the staple features, the generator draw against its probabilities, and
the proposal's symmetry."""
import numpy as np
import pytest


def haar_su3(rng):
    z = (rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))) / np.sqrt(2)
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    return q / np.linalg.det(q) ** (1 / 3)


def random_record(rng, beta=6.0):
    """A staple sum of six SU(3) products near a smooth field and a link."""
    u = haar_su3(rng)
    near = lambda: np.linalg.qr(np.eye(3) + 0.6 * (rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))))[0]
    a = sum(near() @ near() @ near() for _ in range(6)) @ u.conj().T
    return u, a


def m18_of(u, a):
    m = u @ a
    return np.stack([m.real, m.imag], -1).reshape(18).astype(np.float32)


def test_closed_form_rotation_trace(oracle):
    rng = np.random.default_rng(3)
    for _ in range(5):
        u, a = random_record(rng)
        m18 = m18_of(u, a)
        m = m18.astype(np.float64).reshape(9, 2)
        mm = (m[:, 0] + 1j * m[:, 1]).reshape(3, 3)
        for g in range(8):
            for th in (-0.9, -0.2, 0.35, 1.7):
                r = oracle.su3_links(1)
                from ctypes import POINTER, c_double
                oracle.lib().or_su3_generator_rotation(g, c_double(th), r.view(np.float64).ctypes.data_as(POINTER(c_double)))
                f, df = oracle.lp_retr_rotated(g, m18, th)
                assert abs(f - np.trace(r[0] @ mm).real) < 1e-12
                h = 1e-6
                fp, _ = oracle.lp_retr_rotated(g, m18, th + h)
                fm, _ = oracle.lp_retr_rotated(g, m18, th - h)
                assert abs(df - (fp - fm) / (2 * h)) < 1e-7


def _records(rng, n, beta=6.0):
    feats, ms = [], []
    for _ in range(n):
        u, a = random_record(rng, beta)
        feats.append(np.asarray(__import__("oracle").lp_features(a, beta), np.float32))
        ms.append(m18_of(u, a))
    return np.array(feats), np.array(ms)


def _params(rng, scale=0.3):
    p = (rng.standard_normal(6288) * scale).astype(np.float32)
    p[5248 + 9 * 64:5248 + 16 * 64] = 0
    p[6272 + 9:] = 0
    return p


def test_objective_output_gradient(oracle):
    rng = np.random.default_rng(5)
    _, ms = _records(rng, 3)
    for m18 in ms:
        y = rng.standard_normal(16) * 0.7
        e, dy = 0.0, np.zeros(9)
        from ctypes import POINTER, c_double, c_float, byref
        L = oracle.lib()
        ee = c_double()
        L.or_lp_objective(y.ctypes.data_as(POINTER(c_double)), m18.ctypes.data_as(POINTER(c_float)),
                          c_double(6.0), byref(ee), dy.ctypes.data_as(POINTER(c_double)))
        for o in range(9):
            h = 1e-6
            yp, ym = y.copy(), y.copy()
            yp[o] += h
            ym[o] -= h
            ep, em = c_double(), c_double()
            tmp = np.zeros(9)
            L.or_lp_objective(yp.ctypes.data_as(POINTER(c_double)), m18.ctypes.data_as(POINTER(c_float)),
                              c_double(6.0), byref(ep), tmp.ctypes.data_as(POINTER(c_double)))
            L.or_lp_objective(ym.ctypes.data_as(POINTER(c_double)), m18.ctypes.data_as(POINTER(c_float)),
                              c_double(6.0), byref(em), tmp.ctypes.data_as(POINTER(c_double)))
            assert abs(dy[o] - (ep.value - em.value) / (2 * h)) <= 1e-6 * max(1.0, abs(dy[o]))


def test_parameter_gradient_against_finite_differences(oracle):
    rng = np.random.default_rng(11)
    x, m = _records(rng, 6)
    p = _params(rng)
    obj, g = oracle.lp_loss_grad(p, x, m, 6.0, exact=True)
    pd = p.astype(np.float64)
    assert abs(obj - oracle.lp_objective_exact(pd, x, m, 6.0)) < 1e-6
    idx = list(rng.choice(1024, 6, replace=False)) + list(1024 + rng.choice(64, 3, replace=False)) \
        + list(1088 + rng.choice(4096, 6, replace=False)) + list(5248 + rng.choice(9 * 64, 6, replace=False)) \
        + [6272, 6272 + 3, 6272 + 8]
    for i in idx:
        h = 1e-5
        a, b = pd.copy(), pd.copy()
        a[i] += h
        b[i] -= h
        fd = -(oracle.lp_objective_exact(a, x, m, 6.0) - oracle.lp_objective_exact(b, x, m, 6.0)) / (2 * h)
        assert abs(g[i] - fd) <= 2e-5 * max(1e-3, np.abs(g).max()), (i, g[i], fd)
    # the BF16-emulated gradient is the device's; it tracks the exact one
    obj_b, g_b = oracle.lp_loss_grad(p, x, m, 6.0)
    assert abs(obj_b - obj) < 0.05 * abs(obj) + 1e-4
    assert np.linalg.norm(g_b - g) <= 0.05 * np.linalg.norm(g)
    # padding outputs carry no gradient
    assert not np.any(g[5248 + 9 * 64:5248 + 16 * 64]) and not np.any(g[6272 + 9:])


def test_features_gauge_invariant(oracle):
    rng = np.random.default_rng(17)
    for _ in range(4):
        _, a = random_record(rng)
        g, h = haar_su3(rng), haar_su3(rng)
        f0 = oracle.lp_features(a, 5.7)
        f1 = oracle.lp_features(g @ a @ h.conj().T, 5.7)
        assert np.allclose(f0, f1, rtol=1e-10, atol=1e-12)
        assert np.all(np.isfinite(f0)) and 0 <= f0[0] <= 1 and f0[11] <= 1


def test_generator_draw_matches_probabilities(oracle):
    p = np.array([0.05, 0.2, 0.01, 0.3, 0.04, 0.1, 0.15, 0.15])
    counts = np.zeros(8)
    for b in range(2048):
        w = (b << 52) | 12345
        counts[oracle.lp_pick_generator(w, p)] += 1
    assert np.all(np.abs(counts / 2048 - p) <= 1.0 / 2048 + 1e-12)
    # the sign bit and the angle bits do not move the draw
    assert oracle.lp_pick_generator((777 << 52) | (1 << 63), p) == oracle.lp_pick_generator(777 << 52, p)


def test_hit_is_reversible(oracle):
    """The proposal is symmetric: the angle word with the sign bit flipped
    proposes the inverse rotation, which restores the link exactly up to
    rounding, with the same generator and hence the same probability."""
    rng = np.random.default_rng(23)
    u, a = random_record(rng)
    w = int(rng.integers(0, 2 ** 63)) | (1 << 63)
    for g in range(8):
        u1, acc = oracle.su3_hit(u, a, 0.0, 1.3, w, 0, g)        # beta 0: always accepted
        assert acc
        u2, _ = oracle.su3_hit(u1, a, 0.0, 1.3, w ^ (1 << 63), 0, g)
        assert np.abs(u2 - u).max() < 1e-13


def test_proposal_outputs(oracle):
    y = np.zeros(16)
    y[8] = 0.0
    p, s = oracle.lp_proposal(y)
    assert np.allclose(p, 1 / 8) and abs(s - (0.05 + 2.45 * 0.5)) < 1e-15

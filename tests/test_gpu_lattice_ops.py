"""Per-site and per-link lattice queries through the C ABI, against the oracle.

The engine evaluates the reference's Su3Lattice4 / Lattice4 / path_holonomy
methods (path holonomies, Wilson and Polyakov loops, plaquette matrices, the
Wilson action, staples, local actions, gauge transforms, single links) with
the reference's products in the reference's order, so every value here must
equal the oracle's restatement bit for bit; lattice means are held to 1e-12
relative.  Gauge invariance is checked on the device with the reference's
deterministic_su3_site_gauge fixture (su3_lattice.rs:327-340).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXT3 = [4, 4, 4, 6]
EXT2 = [4, 6, 4, 4]


def _su3_field(oracle, ext, seed):
    links = oracle.su3_identity(ext)
    for s in range(3):
        oracle.su3_cb_sweep(ext, links, 0.0, 1.0, seed, s)
    return links


def _su2_field(oracle, ext, seed):
    links = oracle.su2_identity(ext)
    for s in range(2):
        oracle.su2_cb_sweep(ext, links, 0.5, seed, s, 1, 10000)
    return links


def _sites(ext):
    for x0 in range(ext[0]):
        for x1 in range(ext[1]):
            for x2 in range(ext[2]):
                for x3 in range(ext[3]):
                    yield (x0, x1, x2, x3)


# closed paths: a plaquette, rectangles, a path with mixed backward steps,
# and one that winds once around the periodic extent 6 and back
def _closed_paths(oracle):
    return [
        list(oracle.rectangular_path(0, 1, 1, 1)),
        list(oracle.rectangular_path(0, 3, 2, 3)),
        list(oracle.rectangular_path(2, 1, 4, 1)),
        [1, 2, -1, 4, -2, -4, 3, -3],
        [4] * 6 + [-1, 1] + [-4] * 6 + [2, 3, -2, -3],
    ]


@pytest.fixture(scope="module")
def su3(oracle):
    import ymgpu
    links = _su3_field(oracle, EXT3, 11)
    ens = ymgpu.Ensemble([EXT3], 6.0, 1)
    ens.upload(0, links)
    yield ens, links
    ens.close()


@pytest.fixture(scope="module")
def su2(oracle):
    import ymgpu
    links = _su2_field(oracle, EXT2, 12)
    ens = ymgpu.Ensemble([EXT2], 2.3, 1, group=ymgpu.SU2)
    ens.upload(0, links)
    yield ens, links
    ens.close()


def test_su3_wilson_loops_every_site_bitwise(oracle, su3):
    ens, links = su3
    for steps in _closed_paths(oracle):
        got = ens.wilson_loop_sites(0, steps)
        want = np.array([oracle.su3_wilson_loop(EXT3, links, x, steps) for x in _sites(EXT3)])
        assert np.array_equal(got, want), steps
    x = (1, 2, 3, 4)
    steps = _closed_paths(oracle)[3]
    assert ens.wilson_loop(0, x, steps) == oracle.su3_wilson_loop(EXT3, links, x, steps)


def test_su3_open_path_holonomy_bitwise(oracle, su3):
    ens, links = su3
    steps = [1, 4, 4, -3, 2, -1, 4]
    for start in [(0, 0, 0, 0), (3, 1, 2, 5), (2, 3, 0, 1)]:
        hol, end = ens.path_holonomy(0, start, steps)
        want, wend = oracle.su3_path_holonomy(EXT3, links, start, steps)
        assert np.array_equal(hol, want)
        assert end == wend


def test_su3_polyakov_loops_every_site_bitwise(oracle, su3):
    ens, links = su3
    for d in (0, 3):
        got = ens.polyakov_loop_sites(0, d)
        want = np.array([oracle.su3_polyakov_loop(EXT3, links, x, d) for x in _sites(EXT3)])
        assert np.array_equal(got, want)
        assert np.any(got.imag != 0.0)           # the imaginary part is kept
    assert ens.polyakov_loop(0, (1, 1, 2, 3), 3) == oracle.su3_polyakov_loop(EXT3, links, (1, 1, 2, 3), 3)


def test_su3_polyakov_mean_matches_per_site_lines(oracle, su3):
    ens, links = su3
    per = ens.polyakov_loop_sites(0, 3).reshape(EXT3)
    mean = ens.polyakov_loops(3)[0]
    want = per[:, :, :, 0].mean()
    # the mean's kernel multiplies with fma chains, the per-site one without
    assert abs(mean - want) <= 1e-13


def test_su3_plaquette_matrix_and_action_bitwise(oracle, su3):
    ens, links = su3
    for x, mu, nu in [((0, 0, 0, 0), 0, 1), ((3, 2, 1, 5), 2, 3), ((1, 3, 2, 0), 3, 0)]:
        assert np.array_equal(ens.plaquette_at(0, x, mu, nu),
                              oracle.su3_plaquette_matrix(EXT3, links, x, mu, nu))
    for beta in (0.0, 5.7, 6.0):
        assert ens.wilson_action(beta)[0] == oracle.su3_wilson_action(EXT3, links, beta)


def test_su3_action_bitwise_at_8x4(oracle):
    import ymgpu
    ext = [8, 8, 8, 8]
    links = _su3_field(oracle, ext, 21)
    with ymgpu.Ensemble([ext, EXT3], 6.0, [1, 2]) as ens:
        ens.upload(0, links)
        small = _su3_field(oracle, EXT3, 22)
        ens.upload(1, small)
        got = ens.wilson_action(6.0)
    assert got[0] == oracle.su3_wilson_action(ext, links, 6.0)
    assert got[1] == oracle.su3_wilson_action(EXT3, small, 6.0)


def test_su3_local_action_difference_bitwise(oracle, su3):
    ens, links = su3
    rng = np.random.default_rng(5)
    for k in range(12):
        x = tuple(int(rng.integers(0, n)) for n in EXT3)
        mu = int(rng.integers(0, 4))
        rot = oracle.su3_generator_rotation(int(rng.integers(0, 8)), float(rng.uniform(-1, 1)))
        cand = rot @ links[oracle.site_index(EXT3, x) * 4 + mu]
        beta = [0.0, 5.7, 6.0, 12.0][k % 4]
        got = ens.local_action_difference(0, x, mu, cand, beta)
        assert got == oracle.su3_local_action_difference(EXT3, links, x, mu, cand, beta)


def test_su3_local_link_action_is_the_difference(oracle):
    import ymgpu
    links = _su3_field(oracle, EXT3, 13)
    with ymgpu.Ensemble([EXT3], 6.0, 1) as ens:
        ens.upload(0, links)
        x, mu = (2, 1, 3, 4), 2
        cand = oracle.su3_generator_rotation(3, 0.4) @ links[oracle.site_index(EXT3, x) * 4 + mu]
        before = ens.local_link_action(0, x, mu, 6.0)
        diff = ens.local_action_difference(0, x, mu, cand, 6.0)
        ens.set_link(0, x, mu, cand)
        after = ens.local_link_action(0, x, mu, 6.0)
    assert diff == after - before


def test_su3_gauge_transform_bitwise_and_invariance(oracle, su3):
    import ymgpu
    ens, links = su3
    gauges = oracle.su3_deterministic_gauge_field(EXT3)
    want = oracle.su3_gauge_transform(EXT3, links, gauges)
    with ymgpu.Ensemble([EXT3], 6.0, 1) as dst:
        ens.gauge_transform(0, gauges, dst, 0)
        got = dst.download(0)
        assert np.array_equal(got, want)
        # gauge invariance of closed loops, the action and the plaquette
        assert abs(dst.wilson_action(6.0)[0] - ens.wilson_action(6.0)[0]) <= 1e-12 * ens.wilson_action(6.0)[0]
        for steps in _closed_paths(oracle):
            a = dst.wilson_loop_sites(0, steps)
            b = ens.wilson_loop_sites(0, steps)
            assert np.max(np.abs(a - b)) <= 1e-13
        assert abs(dst.average_plaquette()[0] - ens.average_plaquette()[0]) <= 1e-13
        # in place on the same handle gives the same links
        dst.upload(0, links)
        dst.gauge_transform(0, gauges)
        assert np.array_equal(dst.download(0), want)


def test_su3_lattice_mirror(oracle):
    import ymgpu
    links = _su3_field(oracle, EXT3, 14)
    lat = ymgpu.Su3Lattice4.from_links(EXT3, links)
    try:
        x = (1, 2, 3, 4)
        assert np.array_equal(lat.link(x, 2), links[oracle.site_index(EXT3, x) * 4 + 2])
        new = oracle.su3_generator_rotation(0, 0.3) @ lat.link(x, 2)
        lat.set_link(x, 2, new)
        after = lat.links()
        expect = links.copy()
        expect[oracle.site_index(EXT3, x) * 4 + 2] = new
        assert np.array_equal(after, expect)     # one link moved, nothing else touched
        assert lat.wilson_action(6.0) == oracle.su3_wilson_action(EXT3, expect, 6.0)
        assert lat.polyakov_loop(x, 3) == oracle.su3_polyakov_loop(EXT3, expect, x, 3)
        t = lat.gauge_transform(oracle.su3_deterministic_site_gauge)
        assert np.array_equal(t.links(), oracle.su3_gauge_transform(
            EXT3, expect, oracle.su3_deterministic_gauge_field(EXT3)))
        t.close()
        assert ymgpu.su3_ensemble.local_action_difference(lat, x, 2, links[oracle.site_index(EXT3, x) * 4 + 2],
                                                          6.0) == oracle.su3_local_action_difference(
            EXT3, expect, x, 2, links[oracle.site_index(EXT3, x) * 4 + 2], 6.0)
        steps = ymgpu.path_holonomy.rectangular_path(0, 1, 2, 2)
        assert ymgpu.path_holonomy.wilson_loop(lat, x, steps) == oracle.su3_wilson_loop(EXT3, expect, x, steps)
    finally:
        lat.close()


def test_two_row_link_access(oracle):
    import ymgpu
    links = _su3_field(oracle, EXT3, 15)
    with ymgpu.Ensemble([EXT3], 6.0, 1, precision=ymgpu.F32_TWO_ROW) as ens:
        ens.upload(0, links)
        x = (3, 0, 1, 2)
        full = ens.download(0)
        assert np.array_equal(ens.get_link(0, x, 1), full[oracle.site_index(EXT3, x) * 4 + 1])
        ens.set_link(0, x, 1, links[0])
        assert np.array_equal(ens.get_link(0, x, 1), ens.download(0)[0])


def test_query_errors(oracle, su3):
    import ymgpu
    from ymgpu.errors import YmError
    ens, links = su3
    cases = [
        (lambda: ens.wilson_loop(0, (0, 0, 0, 0), [1, 2, -1]), "PathNotClosed"),
        (lambda: ens.wilson_loop_sites(0, []), "EmptyPath"),
        (lambda: ens.wilson_loop(0, (0, 0, 0, 0), [1, 5, -1, -5]), "DirectionOutOfRange"),
        (lambda: ens.wilson_loop(0, (4, 0, 0, 0), [1, -1]), "CoordinateOutOfRange"),
        (lambda: ens.plaquette_at(0, (0, 0, 0, 0), 2, 2), "DirectionsMustDiffer"),
        (lambda: ens.polyakov_loop(0, (0, 0, 0, 6), 3), "CoordinateOutOfRange"),
        (lambda: ens.wilson_action(-1.0), "NegativeBeta"),
        (lambda: ens.wilson_action(float("nan")), "NonFiniteBeta"),
        (lambda: ens.local_action_difference(0, (0, 0, 0, 0), 1, links[1], 12.5), "BetaOutsideReferenceRange"),
        (lambda: ymgpu.path_holonomy.rectangular_path(0, 1, 0, 2), "ZeroRectangleExtent"),
        (lambda: ymgpu.path_holonomy.rectangular_path(1, 1, 1, 2), "DirectionsMustDiffer"),
    ]
    for call, variant in cases:
        with pytest.raises(YmError) as err:
            call()
        assert err.value.variant == variant, (variant, err.value.variant)
    with ymgpu.Ensemble([EXT3], 6.0, 1) as bad:
        bad.upload(0, links)
        bad.set_link(0, (0, 0, 0, 0), 0, 1.001 * links[0])    # outside the 5e-12 gates
        with pytest.raises(YmError) as err:
            bad.plaquette_at(0, (0, 0, 0, 0), 0, 1)
        assert err.value.variant == "NonUnitaryMatrix"
        with pytest.raises(YmError) as err:
            bad.wilson_action(6.0)
        assert err.value.variant == "NonUnitaryMatrix"


def test_su2_loops_every_site_bitwise(oracle, su2):
    ens, links = su2
    for steps in _closed_paths(oracle)[:4]:
        got = ens.wilson_loop_sites(0, steps)
        want = np.array([oracle.su2_wilson_loop(EXT2, links, x, steps) for x in _sites(EXT2)])
        assert np.array_equal(got.real, want) and not np.any(got.imag)
    for d in (1, 3):
        got = ens.polyakov_loop_sites(0, d)
        want = np.array([oracle.su2_polyakov_loop(EXT2, links, x, d) for x in _sites(EXT2)])
        assert np.array_equal(got.real, want)


def test_su2_plaquette_staple_action_bitwise(oracle, su2):
    ens, links = su2
    for x, mu, nu in [((0, 0, 0, 0), 0, 1), ((3, 5, 1, 2), 3, 1)]:
        assert np.array_equal(ens.plaquette_at(0, x, mu, nu), oracle.su2_plaquette(EXT2, links, x, mu, nu))
    for x, mu in [((0, 0, 0, 0), 0), ((2, 4, 3, 1), 2), ((3, 5, 0, 3), 3)]:
        comp, terms = ens.su2_staple(0, x, mu)
        assert np.array_equal(comp, oracle.su2_staple(EXT2, links, x, mu)) and terms == 6
    for beta in (0.0, 2.3):
        assert ens.wilson_action(beta)[0] == oracle.su2_wilson_action(EXT2, links, beta)


def test_su2_lattice_means(oracle):
    import ymgpu
    ext_b = [6, 4, 4, 4]
    la = _su2_field(oracle, EXT2, 31)
    lb = _su2_field(oracle, ext_b, 32)
    with ymgpu.Ensemble([EXT2, ext_b], 2.3, [1, 2], group=ymgpu.SU2) as ens:
        ens.upload(0, la)
        ens.upload(1, lb)
        loops = ens.su2_wilson_loops(4, 3)
        poly = ens.su2_polyakov_loops(0)
    planes = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]
    for ch, (ext, links) in enumerate([(EXT2, la), (ext_b, lb)]):
        for p, (mu, nu) in enumerate(planes):
            for r in range(1, 5):
                for t in range(1, 5):
                    if t > 3:
                        assert loops[ch, p, r - 1, t - 1] == 0.0
                        continue
                    steps = oracle.rectangular_path(mu, nu, r, t)
                    want = np.mean([oracle.su2_wilson_loop(ext, links, x, steps) for x in _sites(ext)])
                    assert abs(loops[ch, p, r - 1, t - 1] - want) <= 1e-12 * max(abs(want), 1e-3)
        lines = [x for x in _sites(ext) if x[0] == 0]
        want = np.mean([oracle.su2_polyakov_loop(ext, links, x, 0) for x in lines])
        assert abs(poly[ch] - want) <= 1e-12 * max(abs(want), 1e-3)


def test_su2_lattice_mirror(oracle):
    import ymgpu
    links = _su2_field(oracle, EXT2, 16)
    lat = ymgpu.Lattice4.from_links(EXT2, links)
    try:
        x = (1, 5, 2, 3)
        assert np.array_equal(lat.link(x, 3), links[oracle.site_index(EXT2, x) * 4 + 3])
        assert lat.rectangular_wilson_loop(x, 1, 2, 3, 2) == oracle.su2_wilson_loop(
            EXT2, links, x, oracle.rectangular_path(1, 2, 3, 2))
        assert lat.polyakov_loop(x, 1) == oracle.su2_polyakov_loop(EXT2, links, x, 1)
        assert lat.wilson_action(2.3) == oracle.su2_wilson_action(EXT2, links, 2.3)
        q = oracle.su2_from_axis_angle([0.0, 0.0, 1.0], 0.4)
        lat.set_link(x, 3, q)
        expect = links.copy()
        expect[oracle.site_index(EXT2, x) * 4 + 3] = q
        assert np.array_equal(lat.links(), expect)
        comp, _ = lat.staple(x, 0)
        assert np.array_equal(comp, oracle.su2_staple(EXT2, expect, x, 0))
    finally:
        lat.close()

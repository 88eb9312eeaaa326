"""Gauge observables and glueball transformations on the B200 vs the oracle.

Bars: per-site holonomies are evaluated as Re Tr of their two half-paths
(each in traversal order) and Polyakov lines as ordered products, so lattice
means agree with the oracle's single-chain, sequential-sum values to
<= 1e-12 relative;
stout smearing and blocking reproduce the reference goldens to 1e-12 and the
oracle's smeared links to 1e-14.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PLANES = [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3)]


def rough(oracle, ext, seed, sweeps=2):
    links = oracle.su3_identity(ext, lift_cap=True)
    for s in range(sweeps):
        oracle.su3_cb_sweep(ext, links, 0.0, 0.6, seed, s)
    return links


def site_iter(ext):
    for x0 in range(ext[0]):
        for x1 in range(ext[1]):
            for x2 in range(ext[2]):
                for x3 in range(ext[3]):
                    yield (x0, x1, x2, x3)


def test_wilson_loops_match_oracle_site_sums(oracle):
    import ymgpu
    ext = [4, 4, 2, 4]
    links = rough(oracle, ext, 41)
    with ymgpu.Ensemble([ext], 6.0, 0) as ens:
        ens.upload(0, links)
        w = ens.wilson_loops(3, 2)[0]
    sites = list(site_iter(ext))
    for p, (mu, nu) in enumerate(PLANES):
        for r in (1, 2, 3):
            for t in (1, 2):
                steps = oracle.rectangular_path(mu, nu, r, t)
                ref = np.mean([oracle.su3_wilson_loop(ext, links, x, steps).real for x in sites])
                assert abs(w[p, r - 1, t - 1] - ref) <= 1e-12 * max(1.0, abs(ref))
    assert np.all(w[:, 3, :] == 0.0) and np.all(w[:, :, 2:] == 0.0)


def test_loops_on_an_uneven_batch(oracle):
    """Chains of different extents in one handle: each chain's Wilson-loop
    and Polyakov-loop means (per-chain tile sums, one thread per Polyakov
    line) match the oracle to 1e-12."""
    import ymgpu
    exts = [[4, 4, 2, 4], [2, 4, 6, 8], [6, 2, 2, 4]]
    starts = [rough(oracle, e, 50 + i) for i, e in enumerate(exts)]
    with ymgpu.Ensemble(exts, 6.0, [1, 2, 3]) as ens:
        for i, st in enumerate(starts):
            ens.upload(i, st)
        w = ens.wilson_loops(2, 2)
        pol = {d: ens.polyakov_loops(d) for d in range(4)}
    for i, e in enumerate(exts):
        sites = list(site_iter(e))
        for p, (mu, nu) in enumerate(PLANES):
            for r in (1, 2):
                for t in (1, 2):
                    steps = oracle.rectangular_path(mu, nu, r, t)
                    ref = np.mean([oracle.su3_wilson_loop(e, starts[i], x, steps).real for x in sites])
                    assert abs(w[i, p, r - 1, t - 1] - ref) <= 1e-12 * max(1.0, abs(ref)), (i, p, r, t)
        for d in range(4):
            ref = np.mean([oracle.su3_polyakov_loop(e, starts[i], x, d) for x in sites if x[d] == 0])
            assert abs(pol[d][i] - ref) <= 1e-12, (i, d)


def test_polyakov_loop_matches_oracle(oracle):
    import ymgpu
    ext = [4, 2, 4, 6]
    links = rough(oracle, ext, 5)
    with ymgpu.Ensemble([ext], 6.0, 0) as ens:
        ens.upload(0, links)
        for d in range(4):
            got = ens.polyakov_loops(d)[0]
            starts = [x for x in site_iter(ext) if x[d] == 0]
            ref = np.mean([oracle.su3_polyakov_loop(ext, links, x, d) for x in starts])
            assert abs(got - ref) <= 1e-12


def test_operator_basis_matches_oracle_and_is_gauge_invariant(oracle):
    import ymgpu
    ext = [4, 4, 4, 6]
    links = rough(oracle, ext, 13)
    g = oracle.su3_deterministic_gauge_field(ext)
    gl = oracle.su3_gauge_transform(ext, links, g)
    with ymgpu.Ensemble([ext, ext], 6.0, 0) as ens:
        ens.upload(0, links)
        ens.upload(1, gl)
        (p0, r0), (p1, r1) = ens.scalar_operator_basis()
    for t in range(ext[3]):
        op, orr, pc, rc = oracle.scalar_a1pp_operator_basis(ext, links, t)
        assert abs(p0[t] - op) <= 1e-12 and abs(r0[t] - orr) <= 1e-12
        assert pc == 3 * 64 and rc == 6 * 64
    assert np.max(np.abs(p0 - p1)) <= 2e-11 and np.max(np.abs(r0 - r1)) <= 2e-11


def test_identity_operator_basis_exact(golden):
    """glueball-operators-phase3a-v1.json: identity -> exactly 1, counts 81/162."""
    import ymgpu
    from ymgpu.glueball import scalar_a1pp_operator_basis
    with ymgpu.Ensemble([[3, 3, 3, 3]], 6.0, 0) as ens:
        for t in range(3):
            b = scalar_a1pp_operator_basis(ens, 0, t)
            assert (b.spatial_plaquette_1x1, b.spatial_rectangle_2x1) == (1.0, 1.0)
            assert (b.plaquette_loop_count, b.rectangle_loop_count) == (81, 162)
        from ymgpu.errors import YmError
        with pytest.raises(YmError) as e:
            scalar_a1pp_operator_basis(ens, 0, 3)
        assert e.value.variant == "TimeSliceOutOfRange"
    for bad, variant in (([2, 3, 3, 3], "SpatialExtentTooSmall"),
                         ([3, 4, 5, 3], "SpatialExtentsNotCubic")):
        with ymgpu.Ensemble([bad], 6.0, 0) as ens:
            with pytest.raises(YmError) as e:
                ens.scalar_operator_basis()
            assert e.value.variant == variant


def test_stout_golden_on_device(oracle, golden):
    """glueball-spatial-stout-phase3b1-v1.json through the device pipeline."""
    import ymgpu
    from ymgpu import glueball as G
    v = [x for x in golden["glueball-spatial-stout-phase3b1-v1.json"]["vectors"]
         if x["id"] == "canonical-nontrivial-fixture-changes-spatial-links"][0]
    ext = v["extents"]
    lat = oracle.su3_identity(ext)
    lat[0] = oracle.su3_traceless_cycle_link()
    with ymgpu.Ensemble([ext], 6.0, 0) as ens:
        ens.upload(0, lat)
        sm = G.spatial_stout_smear(ens, v["rho"], v["levels"])
        got = sm.download(0)
        b = G.scalar_a1pp_operator_basis(sm, 0, 0)
        sm8 = G.spatial_stout_smear(ens, 0.1, 8)
        sm8_links = sm8.download(0)
        sm.close()
        sm8.close()
    tol = v["absolute_tolerance"]
    change = oracle.max_link_residual(ext, lat, got)
    assert abs(change - v["expected"]["maximum_all_link_residual"]) <= tol
    assert abs(b.spatial_plaquette_1x1 - v["expected"]["spatial_plaquette_1x1"]) <= tol
    assert abs(b.spatial_rectangle_2x1 - v["expected"]["spatial_rectangle_2x1"]) <= tol
    ref = oracle.spatial_stout_smear(ext, lat, v["rho"], v["levels"])
    assert np.max(np.abs(got - ref)) <= 1e-14
    u, d = oracle.su3_max_residuals(ext, sm8_links)
    assert u <= 5e-12 and d <= 5e-12


def test_stout_levels_and_errors_match_oracle(oracle):
    import ymgpu
    from ymgpu import glueball as G
    from ymgpu.errors import YmError
    ext = [4, 4, 4, 4]
    lat = rough(oracle, ext, 77)
    with ymgpu.Ensemble([ext], 6.0, 0) as ens:
        ens.upload(0, lat)
        for levels in (0, 1, 3):
            sm = G.spatial_stout_smear(ens, 0.1, levels)
            got = sm.download(0)
            sm.close()
            ref = oracle.spatial_stout_smear(ext, lat, 0.1, levels)
            assert np.max(np.abs(got - ref)) <= 1e-14, levels
            if levels == 0:
                assert np.array_equal(got, lat)
        sm = G.spatial_stout_smear(ens, 0.1, 10, lift_level_cap=True)
        ten = sm.download(0)
        sm.close()
        for rho, lv, variant in ((0.0, 1, "RhoOutOfRange"), (0.250001, 1, "RhoOutOfRange"),
                                 (float("nan"), 1, "NonFiniteRho"), (0.1, 9, "TooManyLevels")):
            with pytest.raises(YmError) as e:
                G.spatial_stout_smear(ens, rho, lv)
            assert e.value.variant == variant
    eight_two = oracle.spatial_stout_smear(ext, oracle.spatial_stout_smear(ext, lat, 0.1, 8), 0.1, 2)
    assert np.max(np.abs(ten - eight_two)) <= 1e-13


def test_block_golden_and_errors(oracle, golden):
    import ymgpu
    from ymgpu import glueball as G
    from ymgpu.errors import YmError
    v = [x for x in golden["glueball-spatial-block-phase3b2-v1.json"]["vectors"]
         if x["id"] == "canonical-coarse-operator-output"][0]
    fext = v["fine_extents"]
    lat = oracle.su3_identity(fext)
    lat[0] = oracle.su3_traceless_cycle_link()
    with ymgpu.Ensemble([fext], 6.0, 0) as ens:
        ens.upload(0, lat)
        co = G.spatial_stride2_block(ens)
        assert list(co.extents[0]) == v["coarse_extents"]
        b = G.scalar_a1pp_operator_basis(co, 0, 0)
        got = co.download(0)
        co.close()
    tol = v["absolute_tolerance"]
    assert abs(b.spatial_plaquette_1x1 - v["expected"]["spatial_plaquette_1x1"]) <= tol
    assert abs(b.spatial_rectangle_2x1 - v["expected"]["spatial_rectangle_2x1"]) <= tol
    _, ref = oracle.spatial_stride2_block(fext, lat)
    assert np.array_equal(got, ref)
    for bad, variant in (([4, 4, 4, 3], "SpatialExtentTooSmall"), ([7, 7, 7, 3], "SpatialExtentNotEven"),
                         ([6, 8, 6, 3], "SpatialExtentsNotCubic")):
        with pytest.raises(YmError) as e:
            G.blocked_extents(bad)
        assert e.value.variant == variant


def test_correlators_from_device_operators_match_oracle(oracle, golden):
    """glueball-connected-correlator-phase3c-v1.json: four shifted-defect
    configurations as four chains of one handle."""
    import ymgpu
    from ymgpu import glueball as G
    v = [x for x in golden["glueball-connected-correlator-phase3c-v1.json"]["vectors"]
         if x["id"] == "shifted-defect-analytic-correlators"][0]
    ext = v["extents"]
    cfgs = []
    for t in range(4):
        lat = oracle.su3_identity(ext)
        lat[oracle.site_index(ext, (0, 0, 0, t)) * 4] = oracle.su3_traceless_cycle_link()
        cfgs.append(lat)
    with ymgpu.Ensemble([ext] * 4, 6.0, 0) as ens:
        for i, l in enumerate(cfgs):
            ens.upload(i, l)
        res = G.scalar_connected_correlators(ens)
    e = v["expected"]
    tol = v["absolute_tolerance"]
    assert abs(res.plaquette_vacuum_mean - e["plaquette_vacuum_mean"]) <= tol
    assert abs(res.rectangle_vacuum_mean - e["rectangle_vacuum_mean"]) <= tol
    assert np.max(np.abs(res.plaquette_connected - e["plaquette_connected"])) <= tol
    assert np.max(np.abs(res.rectangle_connected - e["rectangle_connected"])) <= tol
    assert np.max(np.abs(res.plaquette_raw - e["plaquette_raw"])) <= tol

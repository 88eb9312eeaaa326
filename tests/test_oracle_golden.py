"""Pins the CPU oracle to the reference's golden vectors and known answers.

Every expected value below comes from ``tests/golden/reference_vectors.json``
(copied from the reference's ``test-vectors``) or from a literal the
reference's Rust tests assert; the citing test is named in each docstring.
"""
import math

import numpy as np
import pytest


def vec(golden, file, vid):
    for v in golden[file]["vectors"]:
        if v["id"] == vid:
            return v
    raise KeyError(vid)


def test_splitmix64_stream(oracle, golden):
    """tests/su2_ensemble.rs:33-45 / su2-ensemble-v1.json."""
    v = vec(golden, "su2-ensemble-v1.json", "splitmix64-seed-zero-first-five")
    assert [f"{x:016x}" for x in oracle.splitmix_outputs(0, 5)] == v["outputs_hex"]


def test_su3_stream_seeds(oracle, golden):
    """tests/su3_ensemble.rs:66-73."""
    v = vec(golden, "su3-ensemble-v1.json", "su3-stream-golden-seeds")
    master = int(v["master_seed"], 16)
    got = [f"{oracle.derive_su3_chain_seed(master, c):016x}" for c in v["chain_ids"]]
    assert got == v["derived_seeds_hex"]


def test_su2_chain_seed_identity(oracle):
    """tests/su2_ensemble.rs:48-54."""
    a, b = oracle.derive_chain_seed(7, 0), oracle.derive_chain_seed(7, 1)
    assert a == oracle.derive_chain_seed(7, 0) and a != b


def test_paired_angle_grid(oracle):
    """tests/su3_ensemble.rs:76-88."""
    for raw in [0, 1, 0x000FFFFFFFFFFFFF, 0x123456789ABCDEF0]:
        neg_raw = raw & ~(1 << 63)
        pos_raw = neg_raw | (1 << 63)
        neg = oracle.proposal_angle_from_u64(neg_raw, 0.35)
        pos = oracle.proposal_angle_from_u64(pos_raw, 0.35)
        assert pos == -neg and 0 < pos < 0.35 and -0.35 < neg < 0
    with pytest.raises(oracle.OracleError):
        oracle.proposal_angle_from_u64(5, 0.5e-8)


def test_su3_golden_chain(oracle, golden):
    """tests/su3_ensemble.rs:137-226 / su3-ensemble-v1.json (tolerance 1e-12)."""
    v = vec(golden, "su3-ensemble-v1.json", "frozen-reference-chain-golden-evidence")
    c = v["config"]
    cfg = dict(extents=c["extents"], beta=c["beta"], master_seed=int(c["master_seed"], 16),
               chain_id=c["chain_id"], thermalization_sweeps=c["thermalization_sweeps"],
               measurements=c["measurements"],
               sweeps_between_measurements=c["sweeps_between_measurements"],
               proposal_angle=c["proposal_angle"],
               autocorrelation_max_lag=c["autocorrelation_max_lag"])
    tol = v["floating_absolute_tolerance"]
    _, meas, sc = oracle.su3_run_chain(cfg)
    assert f"{sc.derived_seed:016x}" == v["derived_seed_hex"]
    assert sc.total_sweeps == v["total_sweeps"]
    assert sc.proposals == v["metropolis_proposals"] and sc.accepts == v["metropolis_accepts"]
    assert np.max(np.abs(meas - np.array(v["raw_measurements"]))) <= tol
    d, ac = oracle.diagnostics(meas, c["autocorrelation_max_lag"])
    g = v["diagnostics"]
    assert abs(d.mean - g["mean"]) <= tol
    assert abs(d.variance - g["variance"]) <= tol
    assert np.max(np.abs(ac - np.array(g["autocorrelation"]))) <= tol
    assert d.positive_window_lag == g["positive_window_lag"]
    assert abs(d.integrated_autocorrelation_time - g["integrated_autocorrelation_time"]) <= tol
    assert abs(d.effective_sample_size - g["effective_sample_size"]) <= tol
    assert abs(d.standard_error - g["standard_error"]) <= tol
    assert abs(sc.final_unitarity_residual - v["final_link_unitarity_residual"]) <= tol
    assert abs(sc.final_determinant_residual - v["final_link_determinant_residual"]) <= tol


def test_su3_beta_zero_consumes_two_words(oracle):
    """tests/su3_ensemble.rs:91-106."""
    ext = [2, 2, 2, 2]
    links = oracle.su3_identity(ext)
    seed = oracle.derive_su3_chain_seed(0x3C00198212230101, 0)
    state, p, a = oracle.su3_metropolis_sweep(ext, links, 0.0, 0.35, seed)
    assert p == 64 * 8 and a == p
    ref = oracle.splitmix_outputs(seed, 2 * p + 1)[-1]
    assert oracle.splitmix_outputs(state, 1)[0] == ref


def test_su3_local_delta_matches_full_action(oracle):
    """tests/su3_ensemble.rs:109-124 (|local - full| <= 2e-11)."""
    ext = [2, 2, 2, 2]
    links = oracle.su3_identity(ext)
    coef = np.zeros(8)
    coef[4] = 0.21
    cand = oracle.su3_from_algebra(coef)
    local = oracle.su3_local_action_difference(ext, links, (0, 0, 0, 0), 2, cand, 5.7)
    prop = links.copy()
    prop[2] = cand
    full = oracle.su3_wilson_action(ext, prop, 5.7) - oracle.su3_wilson_action(ext, links, 5.7)
    assert abs(local - full) <= 2e-11


def test_su3_algebra_vectors(oracle, golden):
    """tests/su3_algebra.rs + su3-algebra-v1.json: structure constants and exp."""
    import ctypes as C
    f, d = C.c_double(), C.c_double()
    for (a, b, c), exp_f in [((0, 1, 2), 1.0), ((0, 4, 5), -0.5), ((3, 4, 7), 0.8660254037844386)]:
        oracle.lib().or_su3_structure(a, b, c, C.byref(f), C.byref(d))
        assert abs(f.value - exp_f) <= 2e-15
    for (a, b, c), exp_d in [((0, 0, 7), 0.5773502691896258), ((7, 7, 7), -0.5773502691896258)]:
        oracle.lib().or_su3_structure(a, b, c, C.byref(f), C.byref(d))
        assert abs(d.value - exp_d) <= 2e-15
    coef = np.zeros(8)
    coef[2] = 0.7
    u = oracle.su3_from_algebra(coef)
    exp = np.diag([np.exp(0.35j), np.exp(-0.35j), 1.0])
    assert np.max(np.abs(u - exp)) <= 2e-14


def test_su3_lattice_vectors(oracle, golden):
    """su3-lattice-v1.json: identity action 0, single cycle link action 12 at beta=2."""
    ext = [3, 3, 3, 3]
    lat = oracle.su3_identity(ext)
    assert oracle.su3_wilson_action(ext, lat, 2.0) == 0.0
    lat[0] = oracle.su3_traceless_cycle_link()
    v = vec(golden, "su3-lattice-v1.json", "single-traceless-cycle-link-3x3x3x3-beta2")
    assert abs(oracle.su3_wilson_action(ext, lat, 2.0) - v["expected"]) <= v["tolerance"]
    g = oracle.su3_deterministic_gauge_field(ext)
    tr = oracle.su3_gauge_transform(ext, lat, g)
    assert abs(oracle.su3_wilson_action(ext, tr, 1.7) - oracle.su3_wilson_action(ext, lat, 1.7)) <= 1e-10
    u, d = oracle.su3_max_residuals(ext, tr)
    assert u <= 5e-12 and d <= 5e-12


def test_path_holonomy_vectors(oracle, golden):
    """path-holonomy-v1.json: chair loop on the cycle link, identity rectangle."""
    ext = [3, 3, 3, 3]
    lat = oracle.su3_identity(ext)
    lat[0] = oracle.su3_traceless_cycle_link()
    w = oracle.su3_wilson_loop(ext, lat, (0, 0, 0, 0), [1, 2, 3, -1, -2, -3])
    assert w == 0j
    ext4 = [4, 4, 4, 4]
    idl = oracle.su3_identity(ext4)
    steps = oracle.rectangular_path(0, 3, 2, 3)
    assert oracle.su3_wilson_loop(ext4, idl, (0, 0, 0, 0), steps) == complex(1.0, 0.0)
    g = oracle.su3_deterministic_gauge_field(ext)
    tr = oracle.su3_gauge_transform(ext, lat, g)
    p0 = oracle.su3_polyakov_loop(ext, lat, (0, 0, 0, 0), 0)
    p1 = oracle.su3_polyakov_loop(ext, tr, (0, 0, 0, 0), 0)
    assert abs(p0 - p1) <= 2e-11


def test_su2_observable_vectors(oracle, golden):
    """su2-observables-v1.json / su2-wilson-v1.json (lib.rs:883-891)."""
    ext = [3, 3, 3, 3]
    lat = oracle.su2_identity(ext)
    assert oracle.su2_wilson_action(ext, lat, 2.0) == 0.0
    rect = oracle.rectangular_path(0, 1, 2, 1)
    assert oracle.su2_wilson_loop(ext, lat, (0, 0, 0, 0), rect) == 1.0
    lat[0] = [0.0, 1.0, 0.0, 0.0]
    assert abs(oracle.su2_wilson_action(ext, lat, 2.0) - 12.0) <= 1e-12
    assert abs(oracle.su2_wilson_loop(ext, lat, (0, 0, 0, 0), rect)) <= 1e-12
    assert abs(oracle.su2_polyakov_loop(ext, lat, (0, 0, 0, 0), 0)) <= 1e-12
    st = oracle.su2_staple(ext, lat, (0, 0, 0, 0), 0)
    assert list(st) == [6.0, 0.0, 0.0, 0.0]


def test_su2_heatbath_and_overrelaxation(oracle):
    """tests/su2_ensemble.rs:84-127: invariants and the microcanonical OR check."""
    ext = [2, 2, 2, 2]
    lat = oracle.su2_identity(ext)
    _, _, upd = oracle.su2_heatbath_sweep(ext, lat, 2.3, 1234, 100000)
    assert upd == 64 and oracle.su2_max_unit_residual(ext, lat) <= 1e-12
    lat = oracle.su2_identity(ext)
    oracle.su2_heatbath_sweep(ext, lat, 2.0, 0xFEEDFACECAFEBEEF, 100000)
    before = oracle.su2_wilson_action(ext, lat, 2.0)
    oracle.su2_overrelaxation_sweep(ext, lat)
    after = oracle.su2_wilson_action(ext, lat, 2.0)
    assert abs(after - before) <= 2e-10


def test_su2_beta_zero_haar_band(oracle):
    """tests/su2_ensemble.rs:75-81."""
    cfg = dict(extents=[2, 2, 2, 2], beta=0.0, master_seed=0x0123456789ABCDEF, chain_id=0,
               thermalization_sweeps=1, measurements=64, sweeps_between_measurements=1,
               overrelaxation_sweeps_per_heatbath=1, max_heatbath_attempts_per_link=10000,
               autocorrelation_max_lag=8)
    _, meas, sc = oracle.su2_run_chain(cfg)
    d, _ = oracle.diagnostics(meas, 8)
    assert abs(d.mean) <= 0.12 and d.effective_sample_size >= 8.0
    assert 0.45 <= sc.mean_heatbath_acceptance <= 1.0
    assert sc.final_link_unit_residual <= 1e-12


def test_diagnostics_positive_window(oracle):
    """tests/su2_ensemble.rs:130-137."""
    d, ac = oracle.diagnostics([1.0, -1.0, 1.0, -1.0, 1.0, -1.0], 3)
    assert ac[0] == 1.0 and d.positive_window_lag == 0
    assert d.integrated_autocorrelation_time == 0.5 and d.effective_sample_size == 6.0


def test_sampling_efficiency_vectors(oracle, golden):
    """sampling-efficiency-v1.json / tests/sampling_efficiency.rs:22-70."""
    v = golden["sampling-efficiency-v1.json"]
    tol = v["tolerance"]
    c = v["cost"]
    e = oracle.sampling_efficiency(v["values"], None, v["max_lag"], c["setup"],
                                   c["thermalization"], c["sampling"])
    u = v["unit_weights"]
    assert abs(e.diagnostics.integrated_autocorrelation_time - u["tau_int"]) <= tol
    assert abs(e.combined_ess_proxy - u["combined_ess_proxy"]) <= tol
    assert abs(e.sampling_cost_per_effective_sample_proxy - u["sampling_cost_per_proxy"]) <= tol
    assert abs(e.total_cost_per_effective_sample_proxy - u["total_cost_per_proxy"]) <= tol
    w = v["weights_1_1_1_3"]
    e = oracle.sampling_efficiency(v["values"], np.log([1, 1, 1, 3]), v["max_lag"], c["setup"],
                                   c["thermalization"], c["sampling"])
    assert abs(e.reweighting_efficiency - w["weight_efficiency"]) <= tol
    assert abs(e.weight_only_ess - w["weight_only_ess"]) <= tol
    assert abs(e.total_cost_per_effective_sample_proxy - w["total_cost_per_proxy"]) <= tol
    d, _ = oracle.diagnostics(v["correlated_values"], v["correlated_max_lag"])
    assert abs(d.integrated_autocorrelation_time - v["correlated_tau_int"]) <= tol


def test_operator_basis_vectors(oracle, golden):
    """glueball-operators-phase3a-v1.json."""
    v = vec(golden, "glueball-operators-phase3a-v1.json", "identity-3cubed-spatial-slice")
    ext = v["extents"]
    lat = oracle.su3_identity(ext)
    for t in range(3):
        p, r, pc, rc = oracle.scalar_a1pp_operator_basis(ext, lat, t)
        e = v["expected"]
        assert (p, r, pc, rc) == (e["spatial_plaquette_1x1"], e["spatial_rectangle_2x1"],
                                  e["plaquette_loop_count"], e["rectangle_loop_count"])
    with pytest.raises(oracle.OracleError):
        oracle.scalar_a1pp_operator_basis(ext, lat, 3)


def test_stout_golden(oracle, golden):
    """glueball-spatial-stout-phase3b1-v1.json / glueball_smearing.rs:29-31."""
    v = vec(golden, "glueball-spatial-stout-phase3b1-v1.json",
            "canonical-nontrivial-fixture-changes-spatial-links")
    ext = v["extents"]
    lat = oracle.su3_identity(ext)
    lat[0] = oracle.su3_traceless_cycle_link()
    sm = oracle.spatial_stout_smear(ext, lat, v["rho"], v["levels"])
    tol = v["absolute_tolerance"]
    assert abs(oracle.max_link_residual(ext, lat, sm) - v["expected"]["maximum_all_link_residual"]) <= tol
    p, r, _, _ = oracle.scalar_a1pp_operator_basis(ext, sm, 0)
    assert abs(p - v["expected"]["spatial_plaquette_1x1"]) <= tol
    assert abs(r - v["expected"]["spatial_rectangle_2x1"]) <= tol
    sm8 = oracle.spatial_stout_smear(ext, lat, 0.1, 8)
    u, d = oracle.su3_max_residuals(ext, sm8)
    assert u <= 5e-12 and d <= 5e-12
    assert oracle.max_link_residual(ext, oracle.su3_identity(ext),
                                    oracle.spatial_stout_smear(ext, oracle.su3_identity(ext), 0.1, 3)) == 0.0


def test_block_golden(oracle, golden):
    """glueball-spatial-block-phase3b2-v1.json / glueball_blocking.rs:24-25."""
    v = vec(golden, "glueball-spatial-block-phase3b2-v1.json", "canonical-coarse-operator-output")
    fext = v["fine_extents"]
    lat = oracle.su3_identity(fext)
    lat[0] = oracle.su3_traceless_cycle_link()
    cext, coarse = oracle.spatial_stride2_block(fext, lat)
    assert cext == v["coarse_extents"]
    p, r, _, _ = oracle.scalar_a1pp_operator_basis(cext, coarse, 0)
    tol = v["absolute_tolerance"]
    assert abs(p - v["expected"]["spatial_plaquette_1x1"]) <= tol
    assert abs(r - v["expected"]["spatial_rectangle_2x1"]) <= tol
    for bad in ([4, 4, 4, 3], [7, 7, 7, 3], [6, 8, 6, 3]):
        with pytest.raises(oracle.OracleError):
            oracle.spatial_stride2_block(bad, oracle.su3_identity(bad))


def test_correlator_golden(oracle, golden):
    """glueball-connected-correlator-phase3c-v1.json (tolerance 2e-12)."""
    v = vec(golden, "glueball-connected-correlator-phase3c-v1.json",
            "shifted-defect-analytic-correlators")
    ext = v["extents"]
    cfgs = []
    for t in range(v["configuration_count"]):
        lat = oracle.su3_identity(ext)
        lat[oracle.site_index(ext, (0, 0, 0, t)) * 4] = oracle.su3_traceless_cycle_link()
        cfgs.append(lat)
    vac, raw, con = oracle.scalar_connected_correlators(ext, cfgs)
    e = v["expected"]
    tol = v["absolute_tolerance"]
    assert abs(vac[0] - e["plaquette_vacuum_mean"]) <= tol
    assert abs(vac[1] - e["rectangle_vacuum_mean"]) <= tol
    assert np.max(np.abs(raw[0] - e["plaquette_raw"])) <= tol
    assert np.max(np.abs(raw[1] - e["rectangle_raw"])) <= tol
    assert np.max(np.abs(con[0] - e["plaquette_connected"])) <= tol
    assert np.max(np.abs(con[1] - e["rectangle_connected"])) <= tol


def test_jackknife_replicas_and_covariance(oracle):
    """connected_from_samples (glueball_scalar_production.rs:383-443) equals the
    periodic estimator on the full set; covariance is (n-1)/n scaled."""
    rng = np.random.default_rng(7)
    s = rng.normal(1.0, 0.01, size=(12, 6))
    full = oracle.connected_from_samples(s)
    _, _, con = oracle.periodic_connected_estimator(s)
    assert np.max(np.abs(full - con)) <= 1e-15
    reps = np.stack([oracle.connected_from_samples(s, k) for k in range(12)])
    cov = oracle.jackknife_covariance(reps, 1, 3)
    dev = reps[:, 1:4] - reps[:, 1:4].mean(0)
    assert np.allclose(cov, dev.T @ dev * (11 / 12), rtol=1e-12, atol=1e-18)
    with pytest.raises(oracle.OracleError):
        oracle.jackknife_covariance(reps[:3], 1, 3)


def test_generator_rotation_matches_reference_exponential(oracle):
    """The engine's scalar Taylor chain reproduces su3.rs:409-450 entry for entry."""
    rng = np.random.default_rng(11)
    for g in range(8):
        for th in list(rng.uniform(-1.0, 1.0, 64)) + [0.999999, -0.9, 0.35, 1e-8]:
            coef = np.zeros(8)
            coef[g] = th
            assert np.array_equal(oracle.su3_from_algebra(coef), oracle.su3_generator_rotation(g, th))


def test_staple_action_change_matches_reference(oracle):
    """The engine's staple contraction dS agrees with local_action_difference."""
    ext = [4, 4, 4, 4]
    lat = oracle.su3_identity(ext)
    oracle.su3_cb_sweep(ext, lat, 0.0, 1.0, 99, 0)  # a rough configuration
    rng = np.random.default_rng(3)
    for _ in range(20):
        x = tuple(int(v) for v in rng.integers(0, 4, 4))
        mu = int(rng.integers(0, 4))
        coef = np.zeros(8)
        coef[int(rng.integers(0, 8))] = rng.uniform(-0.3, 0.3)
        cand = oracle.su3_from_algebra(coef) @ lat[oracle.site_index(ext, x) * 4 + mu]
        ref = oracle.su3_local_action_difference(ext, lat, x, mu, cand, 6.0)
        a = oracle.su3_staple(ext, lat, x, mu)
        u = lat[oracle.site_index(ext, x) * 4 + mu]
        ds = 6.0 * (np.trace(u @ a).real - np.trace(cand @ a).real) / 3.0
        assert abs(ds - ref) <= 2e-11


def test_checkerboard_sweep_statistics(oracle):
    """The engine's update order samples the same plaquette as the reference
    order at beta=0 (Haar: <P> = 0) within a loose band."""
    ext = [4, 4, 4, 4]
    lat = oracle.su3_identity(ext)
    for s in range(30):
        oracle.su3_cb_sweep(ext, lat, 0.0, 1.0, 5, s)
    assert abs(oracle.su3_average_plaquette(ext, lat)) < 0.05
    u, d = oracle.su3_max_residuals(ext, lat)
    assert u <= 5e-12 and d <= 5e-12

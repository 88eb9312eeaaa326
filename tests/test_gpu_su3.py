"""SU(3) parity of the CUDA engine against the CPU oracle (runs on a B200).

Bars:
  * reference order replayed on the device: bitwise equal to the oracle and
    to the reference golden chain (tests/su3_ensemble.rs:137-226);
  * checkerboard sweeps: bitwise equal to the oracle's restatement of the
    same update order (or_b200.c) -- candidates, accept decisions, counts;
  * plaquette: <= 1e-12 relative to the reference's sequential sum;
  * residuals: <= 1e-15 absolute of the oracle's maxima.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MASTER = 0x3C00198212230101


def rough_config(oracle, ext, seed, sweeps=3, angle=1.0):
    """A non-trivial SU(3) configuration made by the oracle (beta = 0 sweeps)."""
    links = oracle.su3_identity(ext, lift_cap=True)
    for s in range(sweeps):
        oracle.su3_cb_sweep(ext, links, 0.0, angle, seed, s)
    return links


def test_reference_order_replays_golden_chain(oracle, golden):
    import ymgpu
    v = [x for x in golden["su3-ensemble-v1.json"]["vectors"]
         if x["id"] == "frozen-reference-chain-golden-evidence"][0]
    c = v["config"]
    seed = oracle.derive_su3_chain_seed(int(c["master_seed"], 16), 0)
    with ymgpu.Ensemble([c["extents"]], c["beta"], seed) as ens:
        state, p, a = ens.reference_sweeps(c["proposal_angle"], seed, c["thermalization_sweeps"])
        meas = []
        for _ in range(c["measurements"]):
            state, p, a = ens.reference_sweeps(c["proposal_angle"], state, 1)
            meas.append(ens.reference_average_plaquette()[0])
        gpu_links = ens.download(0)
    assert np.max(np.abs(np.array(meas) - v["raw_measurements"])) <= v["floating_absolute_tolerance"]
    links, ref_meas, _ = oracle.su3_run_chain(dict(
        extents=c["extents"], beta=c["beta"], master_seed=int(c["master_seed"], 16), chain_id=0,
        thermalization_sweeps=c["thermalization_sweeps"], measurements=c["measurements"],
        sweeps_between_measurements=1, proposal_angle=c["proposal_angle"],
        autocorrelation_max_lag=c["autocorrelation_max_lag"]))
    assert np.array_equal(np.array(meas), ref_meas)          # bit for bit
    assert np.array_equal(gpu_links, links)


def test_reference_order_beta_positive_matches_oracle(oracle):
    """beta > 0: accept decisions use exp; equal unless an ulp-borderline draw."""
    import ymgpu
    ext = [2, 2, 2, 4]
    start = rough_config(oracle, ext, 17)
    seed = oracle.derive_su3_chain_seed(MASTER, 3)
    with ymgpu.Ensemble([ext], 5.7, seed) as ens:
        ens.upload(0, start)
        state, p, a = ens.reference_sweeps(0.35, seed, 2)
        gpu = ens.download(0)
    cpu = start.copy()
    st, pp, aa = oracle.su3_metropolis_sweep(ext, cpu, 5.7, 0.35, seed)
    st, pp2, aa2 = oracle.su3_metropolis_sweep(ext, cpu, 5.7, 0.35, st)
    assert int(state[0]) == st and int(a[0]) == aa + aa2
    assert np.array_equal(gpu, cpu)


@pytest.mark.parametrize("uniform", [False, True])
def test_checkerboard_sweeps_bitwise_equal_oracle(oracle, uniform):
    import ymgpu
    ext = [4, 4, 4, 4]
    start = rough_config(oracle, ext, 5)
    seed = oracle.derive_su3_chain_seed(MASTER, 7)
    with ymgpu.Ensemble([ext], 6.0, seed) as ens:
        ens.upload(0, start)
        ens.sweep_index = 11
        ens.metropolis_sweeps(0.3, 3, "uniform" if uniform else "ordered")
        gpu = ens.download(0)
        prop, acc = ens.accounting()
        assert ens.sweep_index == 14
    cpu = start.copy()
    np_, na = 0, 0
    for s in range(11, 14):
        p, a = oracle.su3_cb_sweep(ext, cpu, 6.0, 0.3, seed, s, uniform)
        np_ += p
        na += a
    assert int(prop[0]) == np_ and int(acc[0]) == na
    assert np.array_equal(gpu, cpu)


@pytest.mark.parametrize("uniform", [False, True])
def test_batch_size_does_not_change_a_chain(oracle, uniform):
    """One 4^4 chain alone (128 links per launch) and as one of 120 copies
    with the same seed (15,360 links per launch) ends bit for bit on the
    oracle's result."""
    import ymgpu
    ext = [4, 4, 4, 4]
    start = rough_config(oracle, ext, 6)
    seed = oracle.derive_su3_chain_seed(MASTER, 9)
    mode = "uniform" if uniform else "ordered"
    got = []
    for n in (1, 120):
        with ymgpu.Ensemble([ext] * n, 6.0, [seed] * n) as ens:
            ens.sweep_path = "tiled"
            for k in range(n):
                ens.upload(k, start)
            ens.metropolis_sweeps(0.3, 2, mode)
            got.append((ens.download(0), ens.download(n - 1), int(ens.accounting()[1][0])))
    cpu = start.copy()
    na = 0
    for sw in range(2):
        na += oracle.su3_cb_sweep(ext, cpu, 6.0, 0.3, seed, sw, uniform)[1]
    (a0, _, acc_a), (b0, b1, acc_b) = got
    assert np.array_equal(a0, cpu) and np.array_equal(b0, cpu) and np.array_equal(b1, cpu)
    assert acc_a == acc_b == na


@pytest.mark.parametrize("path", ["tiled", "auto"])
def test_measured_series_survives_a_larger_request(path):
    """A measurement call asking for more rows than the last one grows the
    series buffer; the captured measurement graph must then write into the
    new buffer (every row filled, the last one the lattice's plaquette)."""
    import ymgpu
    with ymgpu.Ensemble([[4, 4, 4, 4]] * 2, 6.0, [3, 4]) as ens:
        ens.sweep_path = path
        ens.metropolis_sweeps(1.0, 20, "uniform")
        first = ens.measured_sweeps(0.3, 5, 1, "uniform")
        second = ens.measured_sweeps(0.3, 40, 1, "uniform")
        last = ens.average_plaquette()
    assert np.all(first > 0.2) and np.all(second > 0.2)
    assert np.array_equal(second[-1], last)


def test_graph_replay_equals_direct_launches(oracle):
    """Batches of >= 8 sweeps replay a captured CUDA graph; the device sweep
    counter advances on every replay, so 20 sweeps (2 replays + 4 direct)
    equal the oracle's sweeps 0..19."""
    import ymgpu
    ext = [4, 4, 4, 6]
    start = rough_config(oracle, ext, 8)
    seed = oracle.derive_su3_chain_seed(MASTER, 21)
    with ymgpu.Ensemble([ext], 5.7, seed) as ens:
        ens.upload(0, start)
        ens.metropolis_sweeps(0.35, 20)
        gpu = ens.download(0)
        assert ens.sweep_index == 20
    cpu = start.copy()
    for s in range(20):
        oracle.su3_cb_sweep(ext, cpu, 5.7, 0.35, seed, s)
    assert np.array_equal(gpu, cpu)


def test_uneven_batch_each_chain_equals_oracle(oracle):
    """Chains of different extents, couplings and seeds in one handle."""
    import ymgpu
    exts = [[4, 4, 4, 4], [2, 4, 6, 8], [6, 6, 6, 2], [4, 4, 4, 10]]
    betas = [6.0, 5.7, 0.0, 6.3]
    seeds = [oracle.derive_su3_chain_seed(MASTER, i) for i in range(4)]
    starts = [rough_config(oracle, e, 30 + i, 2) for i, e in enumerate(exts)]
    with ymgpu.Ensemble(exts, betas, seeds) as ens:
        for i, s in enumerate(starts):
            ens.upload(i, s)
        ens.metropolis_sweeps(0.35, 2)
        gpu = [ens.download(i) for i in range(4)]
        plaq = ens.average_plaquette()
        ures, dres = ens.max_residuals()
    for i, e in enumerate(exts):
        cpu = starts[i].copy()
        for s in range(2):
            oracle.su3_cb_sweep(e, cpu, betas[i], 0.35, seeds[i], s)
        assert np.array_equal(gpu[i], cpu), f"chain {i}"
        ref = oracle.su3_average_plaquette(e, cpu)
        assert abs(plaq[i] - ref) <= 1e-12 * abs(ref)
        u, d = oracle.su3_max_residuals(e, cpu)
        assert abs(ures[i] - u) <= 1e-15 and abs(dres[i] - d) <= 1e-15


def test_plaquette_odd_extents_and_reference_sum(oracle):
    """Measurements accept any extents (lexicographic storage when N3 is odd)."""
    import ymgpu
    exts = [[3, 3, 3, 3], [3, 3, 3, 4], [5, 4, 3, 2]]
    cfgs = []
    for e in exts:
        lat = oracle.su3_identity(e)
        rng = np.random.default_rng(sum(e))
        for l in rng.choice(len(lat), size=len(lat) // 3, replace=False):
            coef = rng.uniform(-0.5, 0.5, 8)
            lat[l] = oracle.su3_from_algebra(coef)
        cfgs.append(lat)
    with ymgpu.Ensemble(exts, 1.0, 0) as ens:
        for i, l in enumerate(cfgs):
            ens.upload(i, l)
            assert np.array_equal(ens.download(i), l)
        plaq = ens.average_plaquette()
        seq = ens.reference_average_plaquette()
    for i, e in enumerate(exts):
        ref = oracle.su3_average_plaquette(e, cfgs[i])
        assert seq[i] == ref                            # sequential order: bit for bit
        assert abs(plaq[i] - ref) <= 1e-12 * abs(ref)


def test_single_traceless_link_and_identity(oracle):
    import ymgpu
    ext = [3, 3, 3, 3]
    lat = oracle.su3_identity(ext)
    with ymgpu.Ensemble([ext], 2.0, 0) as ens:
        assert ens.average_plaquette()[0] == 1.0
        lat[0] = oracle.su3_traceless_cycle_link()
        ens.upload(0, lat)
        p = ens.average_plaquette()[0]
    # one traceless link: 6 of 486 plaquettes have trace 0 -> 1 - 6/486
    assert abs(p - (1.0 - 6.0 / 486.0)) <= 1e-15


def test_fail_closed_paths():
    import ymgpu
    from ymgpu.errors import YmError
    with pytest.raises(YmError) as e:
        ymgpu.Ensemble([[32, 32, 32, 32]], 6.0, 0)
    assert e.value.variant == "LatticeTooLarge"
    with pytest.raises(YmError) as e:
        ymgpu.Ensemble([[4, 1, 4, 4]], 6.0, 0)
    assert e.value.variant == "InvalidLatticeExtent"
    with ymgpu.Ensemble([[3, 3, 3, 4]], 6.0, 0) as ens:
        with pytest.raises(YmError) as e:
            ens.metropolis_sweeps(0.3, 1)
        assert e.value.variant == "NotCheckerboardable"
    with ymgpu.Ensemble([[4, 4, 4, 4]], 13.0, 0) as ens:
        with pytest.raises(YmError) as e:
            ens.metropolis_sweeps(0.3, 1)
        assert e.value.variant == "BetaOutsideReferenceRange"
    with ymgpu.Ensemble([[4, 4, 4, 4]], 6.0, 0) as ens:
        for bad in (0.0, 1.5, float("nan"), 0.5e-8):
            with pytest.raises(YmError) as e:
                ens.metropolis_sweeps(bad, 1)
            assert e.value.variant == "ProposalAngleOutsideReferenceRange"


def test_run_chain_mirror_beta_zero():
    """run_chain through the mirror: beta=0 accepts everything (su3_ensemble.rs:126-134)."""
    from ymgpu.su3_ensemble import Su3EnsembleConfig, run_chain, LINK_RESIDUAL_LIMIT
    cfg = Su3EnsembleConfig([2, 2, 2, 2], 0.0, MASTER, 0, 2, 8, 1, 0.35, 3)
    r = run_chain(cfg)
    assert r.mean_metropolis_acceptance == 1.0
    assert r.metropolis_proposals == 10 * 64 * 8
    assert r.final_link_unitarity_residual <= LINK_RESIDUAL_LIMIT
    r2 = run_chain(cfg)
    assert np.array_equal(r.measurements, r2.measurements)


def test_published_su3_plaquette_statistics(golden):
    """SU(3) 4^4 beta=6.0: the checkerboard sampler reproduces the reference's
    published pooled plaquette (su3-plaquette-baseline-v2.json) within errors."""
    import ymgpu
    from ymgpu.su2_ensemble import diagnostics
    v = golden["su3-plaquette-baseline-v2.json"]
    text = str(v)
    nch = 64
    seeds = [ymgpu.su3_ensemble.derive_su3_chain_seed(0x2C02198105010002, i) for i in range(nch)]
    with ymgpu.Ensemble([[4, 4, 4, 4]] * nch, 6.0, seeds) as ens:
        ens.metropolis_sweeps(0.35, 200)
        series = np.zeros((nch, 200))
        for m in range(200):
            ens.metropolis_sweeps(0.35, 2)
            series[:, m] = ens.average_plaquette()
    means = series.mean(1)
    pooled = means.mean()
    err = means.std(ddof=1) / np.sqrt(nch)
    published, published_err = 0.5992920042685975, 0.0008268453534905
    assert "0.5992920042685975" in text
    assert abs(pooled - published) <= 4.0 * np.hypot(err, published_err)
    d, _ = diagnostics(series[0], 20)
    assert d.effective_sample_size > 5

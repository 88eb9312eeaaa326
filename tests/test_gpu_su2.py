"""SU(2) heat-bath / overrelaxation parity on the B200.

Bars:
  * overrelaxation (pure +,-,*,/,sqrt): bitwise equal to the oracle's
    restatement of the checkerboard order;
  * heat-bath: the reference sampler uses exp_m1, ln_1p, cos and sin, which
    differ between CUDA and glibc by at most a couple of ulps, so a link
    agrees to <= 1e-12 and the attempt counts agree exactly (a draw within an
    ulp of the acceptance bound would flip a decision; never observed);
  * invariants: unit residual <= 1e-12, overrelaxation changes the action by
    <= 2e-10 (tests/su2_ensemble.rs:117-127);
  * statistics: the reference's published SU(2) 10^4 beta=2.3 plaquette
    (docs/PUBLISHED_PLAQUETTE_BASELINE.md: 0.6022919679 +- 0.0004173)
    within 4 combined standard errors, for both samplers.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rough(oracle, ext, seed, beta=1.0):
    links = oracle.su2_identity(ext)
    for s in range(2):
        oracle.su2_cb_sweep(ext, links, beta, seed, s, 1, 100000)
    return links


def cb_overrelax(oracle, ext, links):
    L = oracle.lib()
    L.or_su2_cb_overrelax.argtypes = [C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    assert L.or_su2_cb_overrelax((C.c_int64 * 4)(*ext),
                                 links.ctypes.data_as(C.POINTER(C.c_double))) == 0


def test_overrelaxation_bitwise_equal_oracle(oracle):
    import ymgpu
    ext = [4, 4, 4, 6]
    start = rough(oracle, ext, 3)
    with ymgpu.Ensemble([ext], 2.3, 1, group=ymgpu.SU2) as ens:
        ens.upload(0, start)
        assert np.array_equal(ens.download(0), start)
        ens.overrelaxation_sweeps(2)
        gpu = ens.download(0)
        a0 = oracle.su2_wilson_action(ext, start, 2.0)
        a1 = oracle.su2_wilson_action(ext, gpu, 2.0)
        res = ens.max_unit_residual()[0]
    cpu = start.copy()
    cb_overrelax(oracle, ext, cpu)
    cb_overrelax(oracle, ext, cpu)
    assert np.array_equal(gpu, cpu)
    assert abs(a1 - a0) <= 2e-10
    assert res <= 1e-12


def test_heatbath_matches_oracle_within_ulps(oracle):
    import ymgpu
    ext = [4, 4, 4, 4]
    start = rough(oracle, ext, 9)
    seed = oracle.derive_chain_seed(0x2B0020121116_0101, 0)
    with ymgpu.Ensemble([ext], 2.3, seed, group=ymgpu.SU2) as ens:
        ens.upload(0, start)
        ens.sweep_index = 5
        ens.markov_sweeps(2, overrelaxation_sweeps=1, max_attempts_per_link=10000)
        gpu = ens.download(0)
        prop, upd = ens.heatbath_accounting()
        plaq = ens.average_plaquette()[0]
    cpu = start.copy()
    p = oracle.su2_cb_sweep(ext, cpu, 2.3, seed, 5, 1, 10000)
    p += oracle.su2_cb_sweep(ext, cpu, 2.3, seed, 6, 1, 10000)
    assert int(prop[0]) == p and int(upd[0]) == 2 * len(cpu)
    assert np.max(np.abs(gpu - cpu)) <= 1e-12
    ref = oracle.su2_average_plaquette(ext, cpu)
    assert abs(plaq - ref) <= 1e-12


@pytest.mark.parametrize("sampler", ["reference", "kennedy-pendleton"])
def test_grouped_and_per_thread_kernels_agree(oracle, sampler):
    """Small sub-sweeps run eight lanes per link, large ones one thread per
    link (the switch is at 96 links per SM): the same chain, alone and as one
    of 120 copies with the same seed, ends bit for bit the same."""
    import ymgpu
    ext = [4, 4, 4, 6]
    start = rough(oracle, ext, 21)
    seed = oracle.derive_chain_seed(0x2B0020121116_0101, 3)
    out = []
    for n in (1, 120):
        with ymgpu.Ensemble([ext] * n, 2.3, [seed] * n, group=ymgpu.SU2) as ens:
            for k in range(n):
                ens.upload(k, start)
            ens.markov_sweeps(3, overrelaxation_sweeps=2, max_attempts_per_link=10000, sampler=sampler)
            prop, _ = ens.heatbath_accounting()
            out.append((ens.download(0), ens.download(n - 1), int(prop[0]), int(prop[n - 1])))
    (a0, _, pa, _), (b0, b1, pb0, pb1) = out
    assert np.array_equal(a0, b0) and np.array_equal(a0, b1)
    assert pa == pb0 == pb1


def test_attempt_limit_fails_closed():
    """A bounded sampler that gives up reports HeatbathAttemptLimitExceeded
    (su2_ensemble.rs:229-253) instead of waiting."""
    import ymgpu
    from ymgpu.errors import YmError
    with ymgpu.Ensemble([[4, 4, 4, 4]], 2.3, 11, group=ymgpu.SU2) as ens:
        with pytest.raises(YmError) as e:
            ens.markov_sweeps(1, 0, max_attempts_per_link=1)
        assert e.value.variant == "HeatbathAttemptLimitExceeded"
        ens.markov_sweeps(1, 0, max_attempts_per_link=10000)     # the handle stays usable
        with pytest.raises(YmError) as e:
            ens.markov_sweeps(1, 0, max_attempts_per_link=0)
        assert e.value.variant == "ZeroHeatbathAttemptLimit"
    with ymgpu.Ensemble([[4, 4, 4, 4]], 9.0, 11, group=ymgpu.SU2) as ens:
        with pytest.raises(YmError) as e:
            ens.markov_sweeps(1)
        assert e.value.variant == "BetaOutsideReferenceRange"


def test_beta_zero_haar_band():
    """tests/su2_ensemble.rs:75-81 through the run_chain mirror."""
    from ymgpu.su2_ensemble import EnsembleConfig, run_chain
    cfg = EnsembleConfig((2, 2, 2, 2), 0.0, 0x0123456789ABCDEF, 0, 1, 64, 1, 1, 10000, 8)
    r = run_chain(cfg)
    assert abs(r.diagnostics.mean) <= 0.12
    assert r.diagnostics.effective_sample_size >= 8.0
    assert 0.45 <= r.mean_heatbath_acceptance <= 1.0
    assert r.final_link_unit_residual <= 1e-12


@pytest.mark.parametrize("sampler", ["reference", "kennedy-pendleton"])
def test_published_su2_plaquette(sampler):
    import ymgpu
    from ymgpu.su2_ensemble import derive_chain_seed
    nch = 8
    seeds = [derive_chain_seed(0x2B0020121116_0101, i) for i in range(nch)]
    with ymgpu.Ensemble([[10, 10, 10, 10]] * nch, 2.3, seeds, group=ymgpu.SU2) as ens:
        ens.markov_sweeps(60, 1, sampler=sampler)
        series = np.zeros((nch, 150))
        for m in range(150):
            ens.markov_sweeps(1, 1, sampler=sampler)
            series[:, m] = ens.average_plaquette()
        assert ens.max_unit_residual().max() <= 1e-12
    means = series.mean(1)
    pooled, err = means.mean(), means.std(ddof=1) / np.sqrt(nch)
    published, published_err = 0.6022919679191184, 0.0004173286094490
    assert abs(pooled - published) <= 4.0 * np.hypot(err, published_err)


@pytest.mark.parametrize("sampler", ["reference", "kennedy-pendleton"])
def test_measured_sweeps_equal_separate_calls(sampler):
    """ym_su2_measured_sweeps (one captured graph per measurement) gives the
    series, links and attempt counts of markov_sweeps + average_plaquette
    called one measurement at a time, bit for bit; a later call continues
    the same chain; the attempt limit still fails closed."""
    import ymgpu
    from ymgpu.errors import YmError
    exts = [[4, 4, 4, 6], [6, 4, 4, 4]]
    with ymgpu.Ensemble(exts, 2.3, [21, 22], group=ymgpu.SU2) as a, \
            ymgpu.Ensemble(exts, 2.3, [21, 22], group=ymgpu.SU2) as b:
        got = np.concatenate([a.su2_measured_sweeps(5, 2, 3, sampler=sampler),
                              a.su2_measured_sweeps(4, 2, 3, sampler=sampler)])
        want = []
        for _ in range(9):
            b.markov_sweeps(2, 3, sampler=sampler)
            want.append(b.average_plaquette())
        assert np.array_equal(got, np.array(want))
        for ch in range(2):
            assert np.array_equal(a.download(ch), b.download(ch))
        pa, ua = a.heatbath_accounting()
        pb, ub = b.heatbath_accounting()
        assert np.array_equal(pa, pb) and np.array_equal(ua, ub)
        with pytest.raises(YmError) as e:
            a.su2_measured_sweeps(2, 1, 0, max_attempts_per_link=1, sampler=sampler)
        assert e.value.variant == "HeatbathAttemptLimitExceeded"


def test_measured_sweeps_edge_cases():
    """No measurements is a no-op; an SU(3) handle is the wrong group; a zero
    attempt limit and a negative count are refused before any launch."""
    import ymgpu
    from ymgpu.errors import YmError
    with ymgpu.Ensemble([[4, 4, 4, 4]], 2.3, 5, group=ymgpu.SU2) as ens:
        before = ens.download(0)
        assert ens.su2_measured_sweeps(0).shape == (0, 1)
        assert np.array_equal(before, ens.download(0))
        with pytest.raises(YmError) as e:
            ens.su2_measured_sweeps(1, max_attempts_per_link=0)
        assert e.value.variant == "ZeroHeatbathAttemptLimit"
        assert ymgpu.lib().ym_su2_measured_sweeps(ens.handle, 100, 1, 0, -1, 1, None) != 0
    with ymgpu.Ensemble([[4, 4, 4, 4]], 6.0, 5) as su3:
        with pytest.raises(YmError) as e:
            su3.su2_measured_sweeps(1)
        assert e.value.variant == "WrongGroup"

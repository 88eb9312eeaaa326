"""Batched drivers: the graph-replayed measurement cadence equals direct
launches bit for bit, and the uneven-chain glueball pipeline produces every
correlator surface with the reference's jackknife arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_measured_sweeps_equal_direct_launches():
    import ymgpu
    from ymgpu.su3_ensemble import derive_su3_chain_seed
    seeds = [derive_su3_chain_seed(5, i) for i in range(6)]
    exts = [[4, 4, 4, 4]] * 4 + [[2, 4, 4, 6]] * 2
    with ymgpu.Ensemble(exts, 6.0, seeds) as a, ymgpu.Ensemble(exts, 6.0, seeds) as b:
        s = a.measured_sweeps(0.3, 12, 2, "uniform")
        direct = []
        for _ in range(12):
            b.metropolis_sweeps(0.3, 2, "uniform")
            direct.append(b.average_plaquette())
        assert np.array_equal(s, np.array(direct))
        assert np.array_equal(a.download(5), b.download(5))
        assert a.sweep_index == b.sweep_index == 24
        s2 = a.measured_sweeps(0.3, 3, 2, "uniform")      # the graph is replayed again
        for m in range(3):
            b.metropolis_sweeps(0.3, 2, "uniform")
            assert np.array_equal(s2[m], b.average_plaquette())


def test_batched_chains_driver():
    from ymgpu.pipelines import batched_su3_chains
    r = batched_su3_chains(n_chains=16, measurements=120, thermalization=50)
    assert r.series.shape == (16, 120)
    assert np.all(r.effective_sample_size > 1) and 0.5 < r.acceptance < 1.0
    assert abs(r.pooled_mean - 0.599) < 0.02
    assert r.link_updates == 16 * 1024 * 120


def test_uneven_glueball_pipeline(oracle):
    import ymgpu
    from ymgpu import glueball as G
    from ymgpu.pipelines import scalar_glueball_pipeline
    groups = ((3, (4, 4, 4, 6)), (2, (6, 6, 6, 4)))
    res = scalar_glueball_pipeline(groups, thermalization=6, measurements=2,
                                   sweeps_between_measurements=2, stout_levels=(0, 2))
    keys = {(s.extents, s.stout_levels, s.blocked) for s in res.surfaces}
    assert keys == {((4, 4, 4, 6), 0, False), ((4, 4, 4, 6), 2, False),
                    ((6, 6, 6, 4), 0, False), ((6, 6, 6, 4), 2, False),
                    ((3, 3, 3, 4), 0, True), ((3, 3, 3, 4), 2, True)}
    for s in res.surfaces:
        n_cfg = (3 if s.extents[0] == 4 else 2) * 2
        assert s.plaquette_samples.shape == (n_cfg, s.extents[3])
        assert np.all(np.isfinite(s.plaquette_connected)) and s.plaquette_connected[0] > 0
        assert s.plaquette_jackknife.shape == (n_cfg, s.extents[3])
        # the library's host arithmetic equals the oracle's
        assert np.array_equal(s.plaquette_connected,
                              oracle.connected_from_samples(s.plaquette_samples))
    assert res.link_updates == (3 * 384 + 2 * 864) * 4 * (6 + 2 * 2)


def test_copy_of_consecutive_chains(oracle):
    """ym_ensemble_copy_chains copies a run of chains (uneven extents) in one
    device copy; mismatched extents or ranges fail closed."""
    import ymgpu
    from ymgpu.errors import YmError
    exts = [[4, 4, 4, 4], [2, 4, 6, 8], [4, 4, 2, 6], [4, 4, 4, 4]]
    with ymgpu.Ensemble(exts, 6.0, [1, 2, 3, 4]) as src:
        src.hot_start()
        with ymgpu.Ensemble(exts[1:3], 6.0, [0, 0]) as dst:
            src.copy_chains_to(1, dst, 0, 2)
            assert np.array_equal(dst.download(0), src.download(1))
            assert np.array_equal(dst.download(1), src.download(2))
            with pytest.raises(YmError) as e:
                src.copy_chains_to(0, dst, 0, 2)
            assert e.value.variant == "LatticeExtentsMismatch"
            with pytest.raises(YmError) as e:
                src.copy_chains_to(3, dst, 0, 2)
            assert e.value.variant == "InvalidArgument"
        sub = src.subset([0, 1, 3])
        try:
            for j, c in enumerate([0, 1, 3]):
                assert np.array_equal(sub.download(j), src.download(c))
        finally:
            sub.close()



def test_stout_in_place_continues_levels(oracle):
    """Smearing in place continues the level sequence: 5 + 2 + 3 levels (odd
    counts route through the second buffer) equal 10 levels from scratch
    bit for bit."""
    import ymgpu
    exts = [[4, 4, 4, 6], [6, 6, 6, 4]]
    with ymgpu.Ensemble(exts, 5.7, [1, 2]) as src:
        src.hot_start()
        src.metropolis_sweeps(1.0, 4, "uniform")
        with src.like() as ref, src.like() as inc:
            src.stout_smear_into(ref, 0.1, 10, lift_level_cap=True)
            src.copy_to(inc)
            inc.stout_smear_into(inc, 0.1, 5, lift_level_cap=True)
            inc.stout_smear_into(inc, 0.1, 2, lift_level_cap=True)
            inc.stout_smear_into(inc, 0.1, 3, lift_level_cap=True)
            for c in range(2):
                assert np.array_equal(inc.download(c), ref.download(c))


def test_sweep_layouts_give_the_same_bits_and_the_tuner_picks_one(oracle):
    """Every sub-sweep layout (items of 128, 64 or 32 sites; chain order or
    largest chains first) gives the same links and accept counts on uneven
    chains; the tuner runs on the first call of >= 50 sweeps and reports its
    choice, and its probe sweeps are ordinary sweeps (same bits as a fixed
    layout)."""
    import ymgpu
    from ymgpu.su3_ensemble import derive_su3_chain_seed
    exts = [[4, 4, 4, 10]] * 3 + [[6, 6, 6, 4]] * 2 + [[2, 4, 4, 6]]
    seeds = [derive_su3_chain_seed(9, i) for i in range(len(exts))]
    ref = None
    for item in (128, 64, 32):
        for by_volume in (False, True):
            with ymgpu.Ensemble(exts, 5.7, seeds) as e:
                e.set_sweep_layout(item, by_volume)
                e.metropolis_sweeps(0.35, 5, "ordered")
                e.metropolis_sweeps(0.35, 3, "uniform")
                got = ([e.download(c) for c in range(len(exts))], e.accounting()[1])
                assert e.sweep_layout == {"item_sites": item, "by_volume": by_volume, "tuned": True}
            if ref is None:
                ref = got
            else:
                assert all(np.array_equal(a, b) for a, b in zip(got[0], ref[0]))
                assert np.array_equal(got[1], ref[1])
    with ymgpu.Ensemble(exts, 5.7, seeds) as a, ymgpu.Ensemble(exts, 5.7, seeds) as b:
        assert not a.sweep_layout["tuned"]
        a.metropolis_sweeps(0.35, 100, "ordered")
        assert a.sweep_layout["tuned"] and a.sweep_layout["item_sites"] in (128, 64, 32)
        b.set_sweep_layout(128, False)
        b.metropolis_sweeps(0.35, 100, "ordered")
        for c in range(len(exts)):
            assert np.array_equal(a.download(c), b.download(c))
        assert np.array_equal(a.accounting()[1], b.accounting()[1])


def test_glueball_measurement_graph_equals_separate_calls(oracle):
    """ym_su3_glueball_measure (copy, incremental stout levels, operator
    bases, group blocking, one captured graph) equals the same measurement
    made call by call, bit for bit, on two calls in a row (the second replays
    the graph)."""
    import ymgpu
    from ymgpu import glueball as G
    exts = [[4, 4, 4, 6]] * 2 + [[6, 6, 6, 4]] * 2
    with ymgpu.Ensemble(exts, 5.7, [1, 2, 3, 4]) as ens, ymgpu.Ensemble(exts, 5.7, [1, 2, 3, 4]) as sm:
        ens.hot_start()
        ens.metropolis_sweeps(1.0, 6, "uniform")
        fine = sm.subset([2, 3])
        coarse = fine.like([G.blocked_extents(e) for e in fine.extents])
        ref_sm = ens.like()
        ref_fine = fine.like()
        ref_coarse = coarse.like()
        try:
            for _ in range(2):
                got = ens.glueball_measure(sm, [0, 2, 3], 0.1, [(fine, coarse, 2)])
                ens.copy_to(ref_sm)
                done, want_p, want_r, want_bp, want_br = 0, [], [], [], []
                for lv in (0, 2, 3):
                    if lv > done:
                        ref_sm.stout_smear_into(ref_sm, 0.1, lv - done, lift_level_cap=True)
                        done = lv
                    basis = ref_sm.scalar_operator_basis()
                    want_p.append(np.concatenate([b[0] for b in basis]))
                    want_r.append(np.concatenate([b[1] for b in basis]))
                    ref_sm.copy_subset_to([2, 3], ref_fine)
                    ref_fine.block_into(ref_coarse)
                    cb = ref_coarse.scalar_operator_basis()
                    want_bp.append(np.concatenate([b[0] for b in cb]))
                    want_br.append(np.concatenate([b[1] for b in cb]))
                assert np.array_equal(got[0], np.array(want_p))
                assert np.array_equal(got[1], np.array(want_r))
                assert np.array_equal(got[2], np.array(want_bp))
                assert np.array_equal(got[3], np.array(want_br))
                ens.metropolis_sweeps(0.35, 2, "ordered")
        finally:
            for h in (fine, coarse, ref_sm, ref_fine, ref_coarse):
                h.close()


def test_glueball_prepare_then_measure_equals_measure():
    """ym_su3_glueball_prepare builds and uploads the measurement graph
    without measuring; the measurements after it equal those of a handle that
    was never prepared, bit for bit, and preparing leaves the links alone."""
    import ymgpu
    from ymgpu import glueball as G
    exts = [[4, 4, 4, 6]] * 2 + [[6, 6, 6, 4]] * 2
    with ymgpu.Ensemble(exts, 5.7, [5, 6, 7, 8]) as ens:
        ens.hot_start()
        ens.metropolis_sweeps(1.0, 4, "uniform")
        sms = [ens.like(), ens.like()]
        fines = [sm.subset([2, 3]) for sm in sms]
        coarses = [f.like([G.blocked_extents(e) for e in f.extents]) for f in fines]
        try:
            before = ens.download(0)
            ens.glueball_prepare(sms[0], [0, 1, 3], 0.1, [(fines[0], coarses[0], 2)])
            assert np.array_equal(before, ens.download(0))
            for _ in range(2):
                a = ens.glueball_measure(sms[0], [0, 1, 3], 0.1, [(fines[0], coarses[0], 2)])
                b = ens.glueball_measure(sms[1], [0, 1, 3], 0.1, [(fines[1], coarses[1], 2)])
                for x, y in zip(a, b):
                    assert np.array_equal(x, y)
                ens.metropolis_sweeps(0.35, 1, "ordered")
        finally:
            for h in fines + coarses + sms:
                h.close()

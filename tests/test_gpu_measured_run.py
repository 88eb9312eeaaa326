"""The loop-measurement cadence (ym_su3_measured_run) against the same work
done call by call.

One captured graph per block runs sweeps with the average plaquette after
each, then Wilson loops R x T <= 4 x 4 and Polyakov loops (binary64 through a
converted view for two-row handles).  The series it returns must equal, bit
for bit, the series of the separate entry points (ym_su3_measured_sweeps,
ym_su3_wilson_loops, ym_su3_polyakov_loops, ym_ensemble_convert) replayed
from the same field, seeds and sweep index; and the FP32-versus-FP64
comparison driver must state a first-sweep plaquette error within the FP32
bar (1e-6).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXTS = [[8, 8, 8, 8], [6, 6, 6, 8]]


def _pair(ymgpu, oracle, precision):
    seeds = [oracle.derive_su3_chain_seed(0x5EED, i) for i in range(len(EXTS))]
    a = ymgpu.Ensemble(EXTS, 6.0, seeds, precision=precision)
    b = ymgpu.Ensemble(EXTS, 6.0, seeds, precision=precision)
    a.hot_start()
    a.metropolis_sweeps(1.0, 5, "uniform")
    a.copy_to(b)
    b.sweep_index = a.sweep_index
    return a, b


@pytest.mark.parametrize("two_row", [False, True])
def test_measured_run_equals_separate_calls(oracle, two_row):
    import ymgpu
    prec = ymgpu.F32_TWO_ROW if two_row else ymgpu.F64
    a, b = _pair(ymgpu, oracle, prec)
    va = a.like(precision=ymgpu.F64) if two_row else None
    vb = b.like(precision=ymgpu.F64) if two_row else b
    try:
        blocks, spb = 3, 4
        plaq, wil, pol = a.measured_run(0.3, blocks, spb, 4, 3, 3, "ordered", view=va)
        p_ref, w_ref, l_ref = [], [], []
        for _ in range(blocks):
            p_ref.append(b.measured_sweeps(0.3, spb, 1, "ordered"))
            if two_row:
                b.convert_to(vb)
            w_ref.append(vb.wilson_loops(4, 3))
            l_ref.append(vb.polyakov_loops(3))
        assert np.array_equal(plaq, np.concatenate(p_ref))
        assert np.array_equal(wil, np.stack(w_ref))
        assert np.array_equal(pol, np.stack(l_ref))
        assert np.array_equal(a.download(1), b.download(1))
        assert a.sweep_index == b.sweep_index
        # a second run replays the captured graph and continues the chains
        plaq2, _, _ = a.measured_run(0.3, 1, spb, 4, 3, 3, "ordered", view=va)
        assert np.array_equal(plaq2, b.measured_sweeps(0.3, spb, 1, "ordered"))
    finally:
        for h in (a, b, va) + ((vb,) if two_row else ()):
            if h is not None:
                h.close()


def test_measured_run_rejects_two_row_without_view(oracle):
    import ymgpu
    from ymgpu.errors import YmError
    with ymgpu.Ensemble([EXTS[0]], 6.0, 1, precision=ymgpu.F32_TWO_ROW) as e:
        with pytest.raises(YmError) as err:
            e.measured_run(0.3, 1, 2)
        assert err.value.variant == "NullArgument"
        with ymgpu.Ensemble([[8, 8, 8, 6]], 6.0, 1) as wrong:
            with pytest.raises(YmError) as err:
                e.measured_run(0.3, 1, 2, view=wrong)
            assert err.value.variant == "LatticeExtentsMismatch"


def test_fp32_vs_fp64_comparison(oracle):
    import ymgpu
    from ymgpu.pipelines import fp32_vs_fp64_run
    seeds = [oracle.derive_su3_chain_seed(0x5EED, 7)]
    with ymgpu.Ensemble([[8, 8, 8, 8]], 6.0, seeds) as start:
        start.hot_start()
        start.metropolis_sweeps(1.0, 20, "uniform")
        cmp = fp32_vs_fp64_run(start, n_blocks=3, sweeps_per_block=10)
    assert cmp.fp32.plaquette.shape == (30, 1) and cmp.fp64.wilson.shape == (3, 1, 6, 4, 4)
    assert cmp.first_sweep_plaquette_error <= 1e-6
    assert np.isfinite(cmp.plaquette_combined_sigma) and cmp.plaquette_combined_sigma > 0
    assert cmp.fp32.link_updates == 30 * 8 ** 4 * 4

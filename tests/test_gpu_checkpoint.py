"""Checkpoint and resume: an ensemble restored from its canonical-text
checkpoint continues bit for bit (the streams depend only on seed, sweep
index, site and direction), for SU(3) Metropolis and SU(2) heat-bath +
overrelaxation; two-row FP32 storage is refused."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_su3_checkpoint_resumes_bit_for_bit(tmp_path):
    import ymgpu
    from ymgpu import config as K
    ext = [[4, 4, 4, 6], [6, 4, 4, 4]]
    with ymgpu.Ensemble(ext, [6.0, 5.7], [11, 12]) as ens:
        ens.hot_start()
        ens.metropolis_sweeps(0.3, 3, "ordered")
        path = os.path.join(tmp_path, "su3.ckpt")
        K.save_checkpoint(ens, path)
        ens.metropolis_sweeps(0.3, 3, "ordered")
        straight = [ens.download(k) for k in range(2)]
        idx = ens.sweep_index
    with K.load_checkpoint(path) as back:
        assert back.extents == [tuple(e) for e in ext]
        assert list(back.beta) == [6.0, 5.7] and list(back.seeds) == [11, 12]
        back.metropolis_sweeps(0.3, 3, "ordered")
        assert back.sweep_index == idx
        for k in range(2):
            assert np.array_equal(back.download(k), straight[k])


def test_su2_checkpoint_resumes_bit_for_bit(tmp_path):
    import ymgpu
    from ymgpu import config as K
    with ymgpu.Ensemble([[4, 4, 4, 4]] * 2, 2.3, [21, 22], group=ymgpu.SU2) as ens:
        ens.markov_sweeps(2, 1)
        path = os.path.join(tmp_path, "su2.ckpt")
        K.save_checkpoint(ens, path)
        ens.markov_sweeps(2, 1)
        straight = [ens.download(k) for k in range(2)]
    text = open(path).read()
    assert "\nYM-SU2-CONFIG-V1\nextents=4,4,4,4\nlink_count=1024\n" in text
    with K.load_checkpoint(path) as back:
        back.markov_sweeps(2, 1)
        for k in range(2):
            assert np.array_equal(back.download(k), straight[k])


def test_two_row_storage_is_refused(tmp_path):
    import ymgpu
    from ymgpu import config as K
    from ymgpu.errors import YmError
    with ymgpu.Ensemble([[4, 4, 4, 4]], 6.0, [3], precision=ymgpu.F32_TWO_ROW) as ens:
        with pytest.raises(YmError) as e:
            K.save_checkpoint(ens, os.path.join(tmp_path, "x"))
        assert e.value.variant == "UnsupportedPrecision"

"""Two handles driven from two host threads at once (each with its own CUDA
stream; the ctypes calls release the interpreter lock) give the same bits
as the same calls made one handle after the other."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EXT = [[8, 8, 8, 8]]


def _cycle(ens, host, steps):
    plaq = []
    for _ in range(steps):
        ens.upload(0, host)
        ens.metropolis_sweeps(0.3, 1, "ordered")
        plaq.append(float(ens.average_plaquette()[0]))
        ens.download(0, host)
    return plaq


def _start(seed):
    import ymgpu
    ens = ymgpu.Ensemble(EXT, 6.0, seed)
    ens.hot_start()
    host = ens.download(0)
    return ens, host


def test_two_threads_equal_sequential():
    seeds, steps = [11, 12], 6
    seq = []
    for sd in seeds:
        ens, host = _start(sd)
        try:
            seq.append((_cycle(ens, host, steps), host.copy()))
        finally:
            ens.close()
    handles = [_start(sd) for sd in seeds]
    out = [None, None]

    def run(i):
        ens, host = handles[i]
        out[i] = (_cycle(ens, host, steps), host)

    try:
        threads = [threading.Thread(target=run, args=(i,)) for i in range(2)]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
    finally:
        for ens, _ in handles:
            ens.close()
    for (p_seq, l_seq), (p_thr, l_thr) in zip(seq, out):
        assert p_seq == p_thr
        assert np.array_equal(l_seq, l_thr)

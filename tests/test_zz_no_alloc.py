"""The allocation-free average plaquette (ym_su3_average_plaquette_noalloc).

It exists for callers that cannot allocate device memory -- a framework whose
pool owns the GPU and only lends out buffers it allocated, or a deployment
that must keep a fixed device footprint after start-up.  Called through the
C ABI with device buffers the test allocates (the entry point allocates
nothing), its result must equal the allocating entry point's
(ym_average_plaquette) and the oracle's sequential sum within the plaquette
tolerance of the other tests, 1e-12 relative, on two calls in a row, and the
device's free memory must not move across a call.  This file is collected
last so a run that stops at the first failure has already run every other
test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rough(oracle, ext, seed):
    links = oracle.su3_identity(ext)
    for s in range(2):
        oracle.su3_cb_sweep(ext, links, 0.0, 1.0, seed, s)
    return links


def _noalloc(torch, ext, links):
    import ymgpu
    d_links = torch.from_numpy(links.view(np.float64).reshape(-1).copy()).cuda()
    d_out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    e = (C.c_int64 * 4)(*ext)
    stream = torch.cuda.current_stream().cuda_stream
    st = ymgpu.lib().ym_su3_average_plaquette_noalloc(C.c_void_p(d_links.data_ptr()), e,
                                                      C.c_void_p(d_out.data_ptr()),
                                                      C.c_void_p(stream))
    assert st == 0
    torch.cuda.synchronize()
    return float(d_out.item())


def test_noalloc_plaquette_equals_allocating_entry_point(oracle):
    torch = pytest.importorskip("torch")
    import ymgpu
    ext = [8, 8, 8, 6]
    first = _rough(oracle, ext, 3)
    second = _rough(oracle, ext, 4)
    with ymgpu.Ensemble([ext], 6.0, 1) as ens:
        ens.upload(0, first)
        ref1 = float(ens.average_plaquette()[0])
        ens.upload(0, second)
        ref2 = float(ens.average_plaquette()[0])
    got1 = _noalloc(torch, ext, first)
    got2 = _noalloc(torch, ext, second)       # second call in a row reuses the scratch
    assert abs(got1 - ref1) <= 1e-12 * abs(ref1)
    assert abs(got2 - ref2) <= 1e-12 * abs(ref2)
    for got, links in ((got1, first), (got2, second)):
        want = oracle.su3_average_plaquette(ext, links)
        assert abs(got - want) <= 1e-12 * abs(want)
    assert got1 != got2


def test_noalloc_plaquette_takes_no_device_memory(oracle):
    torch = pytest.importorskip("torch")
    import ymgpu
    ext = [8, 8, 8, 6]
    links = _rough(oracle, ext, 5)
    d_links = torch.from_numpy(links.view(np.float64).reshape(-1).copy()).cuda()
    d_out = torch.zeros(1, dtype=torch.float64, device="cuda")
    e = (C.c_int64 * 4)(*ext)
    fn = ymgpu.lib().ym_su3_average_plaquette_noalloc
    assert fn(C.c_void_p(d_links.data_ptr()), e, C.c_void_p(d_out.data_ptr()), None) == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert fn(C.c_void_p(d_links.data_ptr()), e, C.c_void_p(d_out.data_ptr()), None) == 0
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    want = oracle.su3_average_plaquette(ext, links)
    assert abs(float(d_out.item()) - want) <= 1e-12 * abs(want)


def test_noalloc_rejects_lattices_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    import ymgpu
    from ymgpu.errors import VARIANTS
    d = torch.zeros(2, dtype=torch.float64, device="cuda")
    e = (C.c_int64 * 4)(64, 64, 64, 64)            # 16.7M sites > 8,388,608
    st = ymgpu.lib().ym_su3_average_plaquette_noalloc(C.c_void_p(d.data_ptr()), e,
                                                      C.c_void_p(d.data_ptr()), None)
    assert st == VARIANTS["ScratchTooSmall"]

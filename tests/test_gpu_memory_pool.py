"""Handles draw device memory from the device's memory pool, which keeps what
destroyed handles free; ym_device_release_pooled_memory gives it back."""
import pytest

pytestmark = pytest.mark.gpu


def test_pooled_memory_is_reused_and_released():
    torch = pytest.importorskip("torch")
    import ymgpu
    ext = [[32, 32, 32, 32]]
    ymgpu.release_pooled_memory(0)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    with ymgpu.Ensemble(ext, 6.0, 1, lift_reference_caps=True) as a:
        a.hot_start()
        first = a.average_plaquette()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 >= 1_000_000_000          # 1.2 GB of links and staging stay pooled
    with ymgpu.Ensemble(ext, 6.0, 1, lift_reference_caps=True) as b:   # served from the pool
        b.hot_start()
        assert (b.average_plaquette() == first).all()
        free2, _ = torch.cuda.mem_get_info()
        assert free2 >= free1 - 64 * 2**20
    ymgpu.release_pooled_memory(0)
    free3, _ = torch.cuda.mem_get_info()
    assert free3 >= free0 - 64 * 2**20
    from ymgpu.errors import YmError
    with pytest.raises(YmError):
        ymgpu.release_pooled_memory(10**6)

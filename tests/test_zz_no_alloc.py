"""The closest-hit entry point that allocates no memory.

Some callers of this library cannot call cudaMalloc when they query rays:
their host application owns the device-memory budget through its own pools,
or the query runs on a per-frame path that cannot take an allocation's
implicit synchronisation or a late out-of-memory failure.
alpine_gpu_trace_noalloc serves them from one fixed staging array in device
memory.

This test calls it through the C ABI twice in a row, with different rays,
before any ordinary query has grown the context's own staging buffers. It
checks that the device's free memory does not change across those calls (the
property the entry point exists for; the first call on a device may load the
module that holds the array, so a warm-up call comes before the first
reading). Then it checks each result against the ordinary alpine_gpu_trace
bit-exactly (the tolerance of every traversal test here), and that a batch
beyond the fixed maximum is rejected with a clear error. The file is named to
be collected last.
"""
import numpy as np
import pytest

from alpine_b200 import gpu, scenes

pytestmark = pytest.mark.gpu


def _free_bytes():
    import torch

    torch.cuda.synchronize(0)
    return torch.cuda.mem_get_info(0)[0]


def test_noalloc_matches_trace_on_two_calls():
    _free_bytes()  # initialises the runtime's view of the device first
    ctx = gpu.Context(0)
    try:
        verts, idx = scenes.triangle_soup(50000, seed=71, mu=np.log(0.01))
        ctx.add_mesh(verts, idx)
        ctx.build()
        first = np.concatenate([scenes.primary_rays(128, 128), scenes.incoherent_rays(40000, seed=72)])
        second = scenes.incoherent_rays(gpu.NOALLOC_MAX_RAYS, seed=73)
        ctx.trace_noalloc(scenes.incoherent_rays(1024, seed=70))  # warm-up: per-device set-up
        free_before = _free_bytes()
        results = [ctx.trace_noalloc(rays) for rays in (first, second)]
        free_after = _free_bytes()
        assert free_after == free_before, f"device free memory changed by {free_before - free_after} bytes"
        for rays, a in zip((first, second), results):
            b = ctx.trace(rays)
            assert a.tobytes() == b.tobytes()
            assert (a["prim"] != gpu.MISS).sum() > 1000
        too_many = scenes.incoherent_rays(gpu.NOALLOC_MAX_RAYS + 1, seed=74)
        with pytest.raises(gpu.GpuError) as e:
            ctx.trace_noalloc(too_many)
        assert e.value.code == gpu.ERR_INVALID_ARGUMENT and "65536" in str(e.value)
    finally:
        ctx.close()

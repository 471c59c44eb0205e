"""nova_b200_render_noalloc: the allocation-free render entry point.

It is for callers that cannot call cudaMalloc while they render: a host loop whose device memory is
entirely reserved by another allocator (a framework's caching allocator that has claimed the GPU),
or a real-time loop that must not risk an allocation failure mid-frame.  Its film must agree with
nova_b200_render's for the same sample range (within rtol 1e-5 / atol 1e-6, the two paths compile
the same device functions into different kernels) and with the oracle (rel. RMSE <= 1e-3), on two
calls in a row (the second call reuses the shared static scratch array), and the calls must leave
the device's free memory unchanged.

This file sorts last so that a run stopping at the first failure has already run every other test.
"""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

pytestmark = pytest.mark.gpu

RTOL, ATOL, REL_RMSE = 1e-5, 1e-6, 1e-3


def _rel_rmse(got, ref):
    d = (got[..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(ref[..., :3], 1e-3)
    return float(np.sqrt(np.mean(d * d)))


def _oracle_range(scene, W, H, spp, depth, begin, count, seed, rr_start):
    """The oracle's mean over samples [begin, begin + count) of every pixel, in sample order."""
    import oracle_binding
    osc = oracle_binding.OracleScene(scene)
    opt = oracle_binding.options(W, H, spp, depth, seed=seed, rr_start=rr_start)
    ys, xs = np.mgrid[0:H, 0:W]
    acc = np.zeros((H * W, 3), np.float32)
    for s in range(begin, begin + count):
        acc += osc.sample_radiance(opt, xs.reshape(-1), ys.reshape(-1), np.full(H * W, s))
    return (acc / np.float32(count)).reshape(H, W, 3)


def test_noalloc_render_matches_render_and_oracle_twice_without_allocating():
    import torch
    from axomae_b200 import native, scenes
    assert torch.cuda.is_available()
    W, H, spp, depth, seed = 72, 40, 32, 6, 1
    scene = scenes.mixed_scene(20000, W, H, seed=9)
    ctx = native.Context(0)
    try:
        ctx.upload(scene)
        ctx.build()
        ranges = ((0, 8), (8, 24))
        refs = []
        for begin, count in ranges:
            frame = native.make_frame(scene, W, H, spp, depth, seed=seed, sample_begin=begin, sample_count=count,
                                      rr_start=3, reset=1)
            ref = np.zeros((H, W, 4), np.float32)
            ctx.render(frame, film_host=ref)
            refs.append(ref)
        outs = [torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda") for _ in ranges]
        torch.cuda.synchronize()  # the fills run on torch's stream, the render on the context's
        free = [torch.cuda.mem_get_info(0)[0]]
        for (begin, count), out in zip(ranges, outs):
            frame = native.make_frame(scene, W, H, spp, depth, seed=seed, sample_begin=begin, sample_count=count,
                                      rr_start=3, reset=1)
            ctx.render_noalloc(frame, out.data_ptr())
            free.append(torch.cuda.mem_get_info(0)[0])
        assert free[1] == free[0] and free[2] == free[0], "free device memory changed: %s" % free
        for (begin, count), out, ref in zip(ranges, outs, refs):
            got = out.cpu().numpy()
            assert np.isfinite(got).all()
            np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL)
            orc = _oracle_range(scene, W, H, spp, depth, begin, count, seed, 3)
            assert _rel_rmse(got, orc) <= REL_RMSE
    finally:
        ctx.close()


def test_noalloc_frame_split_into_uneven_chunks():
    """256 x 200 pixels x 48 samples = 2,457,600 paths: more than the 2 Mi-path scratch, so the call
    renders a 43,690-pixel chunk and a 7,510-pixel one."""
    import torch
    from axomae_b200 import native, scenes
    W, H, spp, depth = 256, 200, 48, 4
    scene = scenes.spheres_scene(W, H, n_spheres=16)
    ctx = native.Context(0)
    try:
        ctx.upload(scene)
        ctx.build()
        frame = native.make_frame(scene, W, H, spp, depth, seed=3)
        ref = np.zeros((H, W, 4), np.float32)
        ctx.render(frame, film_host=ref)
        out = torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        ctx.render_noalloc(frame, out.data_ptr())
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL)
    finally:
        ctx.close()


def test_noalloc_first_call_succeeds_with_device_memory_full():
    """Everything the call needs is taken when the context is created: with all but a few MiB of
    device memory held by torch (less than the 32 MiB scratch), the first call still renders."""
    import torch
    from axomae_b200 import native, scenes
    W, H, spp, depth = 48, 32, 8, 4
    scene = scenes.spheres_scene(W, H, n_spheres=8)
    ctx = native.Context(0)
    hog = []
    try:
        ctx.upload(scene)
        ctx.build()
        out = torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        for step in (1 << 30, 64 << 20, 2 << 20):
            while True:
                try:
                    hog.append(torch.empty(step, dtype=torch.uint8, device="cuda"))
                except torch.OutOfMemoryError:
                    break
        for _ in range(4):  # hand back up to 8 MiB of the smallest blocks so the runtime's own bookkeeping
            if hog and hog[-1].numel() == (2 << 20):  # is not starved (never a large block: that would
                hog.pop()                             # leave more than the scratch free)
        torch.cuda.empty_cache()
        left = torch.cuda.mem_get_info(0)[0]
        assert left < (32 << 20), "could not fill device memory (%d bytes left)" % left
        frame = native.make_frame(scene, W, H, spp, depth)
        ctx.render_noalloc(frame, out.data_ptr())
        got = out.cpu().numpy()
        hog.clear()
        torch.cuda.empty_cache()
        ref = np.zeros((H, W, 4), np.float32)
        ctx.render(frame, film_host=ref)
        np.testing.assert_allclose(got, ref, rtol=RTOL, atol=ATOL)
    finally:
        hog.clear()
        torch.cuda.empty_cache()
        ctx.close()


def test_noalloc_rejects_oversized_sample_range():
    import torch
    from axomae_b200 import native, scenes
    scene = scenes.spheres_scene(8, 8, n_spheres=2)
    ctx = native.Context(0)
    try:
        ctx.upload(scene)
        ctx.build()
        out = torch.zeros((1, 1, 4), dtype=torch.float32, device="cuda")
        with pytest.raises(native.NovaError) as e:
            ctx.render_noalloc(native.make_frame(scene, 1, 1, 3000000, 2, sample_count=2200000), out.data_ptr())
        assert e.value.status == 15 and "scratch limit" in str(e.value)
    finally:
        ctx.close()

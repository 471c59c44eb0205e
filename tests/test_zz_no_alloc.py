"""nova_b200_render_noalloc: the allocation-free render entry point, for callers that cannot call
cudaMalloc during a frame (device memory fully reserved by another allocator, or a real-time loop
that must not risk an allocation).  Its output must equal nova_b200_render's for the same sample
range, on two calls in a row (the second call reuses the shared static scratch array).

This file sorts last so that a run stopping at the first failure has already run every other test.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_render_matches_render_twice():
    import torch
    from axomae_b200 import native, scenes
    assert torch.cuda.is_available()
    scene = scenes.mixed_scene(20000, 72, 40, seed=9)
    ctx = native.Context(0)
    try:
        ctx.upload(scene)
        ctx.build()
        W, H = 72, 40
        for begin, count in ((0, 8), (8, 24)):
            frame = native.make_frame(scene, W, H, 32, 6, seed=1, sample_begin=begin, sample_count=count,
                                      rr_start=3, reset=1)
            ref = np.zeros((H, W, 4), np.float32)
            ctx.render(frame, film_host=ref)
            out = torch.full((H, W, 4), float("nan"), dtype=torch.float32, device="cuda")
            ctx.render_noalloc(frame, out.data_ptr())
            got = out.cpu().numpy()
            assert np.isfinite(got).all()
            d = (got[..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(ref[..., :3], 1e-3)
            assert float(np.sqrt(np.mean(d * d))) <= 1e-3
            np.testing.assert_allclose(got, ref, rtol=1e-5, atol=1e-6)
    finally:
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

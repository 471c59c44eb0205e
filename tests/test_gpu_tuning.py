"""Launch tuning and the autotuner: tunings change speed, never a result bit."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def scene_ctx():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    from axomae_b200 import native, scenes
    s = scenes.mixed_scene(20000, 61, 47, seed=9)
    c = native.Context(0)
    c.upload(s)
    c.build()
    yield s, c
    c.close()


def _film(c, s, W=61, H=47, spp=32, depth=6):
    from axomae_b200 import native
    film = np.zeros((H, W, 4), np.float32)
    st = c.render(native.make_frame(s, W, H, spp, depth), film_host=film)
    return film, st


@pytest.mark.parametrize("tuning", [
    dict(queue_capacity=65536),                                # many small waves
    dict(trace_block=32, shade_block=96),
    dict(tile_w=8, tile_h=4),
    dict(tile_w=16, tile_h=2, queue_capacity=1 << 20, trace_block=64, shade_block=64),
    dict(tile_w=64, tile_h=64),                                # tiles larger than the frame's last row / column
    dict(tile_w=1, tile_h=1),                                  # image rows
    dict(trace_mode=1),                                        # persistent trace warps
    dict(trace_mode=1, queue_capacity=65536, tile_w=8, tile_h=4),
    dict(trace_mode=2),                                        # counting node visits and triangle tests
], ids=["small-waves", "blocks", "tile8x4", "mixed", "tile64", "rows", "persistent", "persistent-small-waves",
        "counting"])
def test_tuning_does_not_change_results(scene_ctx, tuning):
    s, c = scene_ctx
    c.set_tuning()
    ref, st0 = _film(c, s)
    c.set_tuning(**tuning)
    try:
        out, st1 = _film(c, s)
    finally:
        c.set_tuning()
    assert np.array_equal(out, ref)
    assert st1.traced == st0.traced
    if tuning.get("queue_capacity") == 65536:
        assert st1.waves > st0.waves
    if tuning.get("trace_mode") == 2:  # at least the root per ray; a triangle test for most rays
        assert st1.node_visits >= st1.traced and 0 < st1.tri_tests < 64 * st1.traced
    else:
        assert st1.node_visits == 0 and st1.tri_tests == 0


def test_invalid_tuning_rejected(scene_ctx):
    from axomae_b200 import native
    _, c = scene_ctx
    for bad in (dict(queue_capacity=100), dict(trace_block=256), dict(tile_w=8), dict(tile_w=5, tile_h=5),
                dict(trace_mode=7)):
        with pytest.raises(native.NovaError) as e:
            c.set_tuning(**bad)
        assert e.value.status == 15
    assert c.get_tuning().queue_capacity == 0


def test_autotune_applies_and_caches(tmp_path):
    from axomae_b200 import native, scenes
    specs = [(scenes.mixed_scene(15000, 40, 40, seed=1), 40, 40, 4, 6),
             (scenes.spheres_scene(32, 24, n_spheres=6, seed=2), 32, 24, 8, 4)]
    ctxs = []
    try:
        frames, refs = [], []
        for s, W, H, spp, depth in specs:
            c = native.Context(0)
            ctxs.append(c)
            c.upload(s)
            c.build()
            fr = native.make_frame(s, W, H, spp, depth)
            frames.append(fr)
            ref = np.zeros((H, W, 4), np.float32)
            c.render(fr, film_host=ref)
            refs.append(ref)
        cache = tmp_path / "tune.txt"
        t = native.autotune(ctxs, frames, str(cache), flags=native.TUNE_BVH_WIDTH)
        assert t.bvh_width in (2, 8)
        lines = cache.read_text().strip().splitlines()
        assert len(lines) == 1 and len(lines[0].split()) == 8
        for c in ctxs:
            got = c.get_tuning()
            assert (got.queue_capacity, got.trace_block, got.shade_block, got.tile_w, got.tile_h) == (
                t.queue_capacity, t.trace_block, t.shade_block, t.tile_w, t.tile_h)
            assert got.bvh_width == t.bvh_width
        outs = [np.zeros_like(r) for r in refs]
        native.render_batch(ctxs, frames, films_host=outs)
        for c, fr, o, r in zip(ctxs, frames, outs, refs):
            single = np.zeros_like(r)
            c.render(fr, film_host=single)
            assert np.array_equal(o, single)
            if t.bvh_width == 2:
                assert np.array_equal(o, r)
            else:  # the 8-wide BVH may report the other of two triangles at exactly equal distance
                assert np.abs(o - r).max() <= 1e-3 * max(1.0, float(np.abs(r).max())) or \
                    np.mean(np.abs(o - r) > 0) < 1e-3
        # a second call finds the cached entry
        t2 = native.autotune(ctxs, frames, str(cache), flags=native.TUNE_BVH_WIDTH)
        assert t2.as_dict() == t.as_dict()
        assert len(cache.read_text().strip().splitlines()) == 1
    finally:
        for c in ctxs:
            c.close()

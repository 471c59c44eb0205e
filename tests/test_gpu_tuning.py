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
    dict(trace_mode=3),                                        # persistent wavefront: one launch per chunk
    dict(trace_mode=3, queue_capacity=65536, tile_w=8, tile_h=4),
    dict(trace_mode=3, bvh_width=1),
], ids=["small-waves", "blocks", "tile8x4", "mixed", "tile64", "rows", "persistent", "persistent-small-waves",
        "counting", "wavefront", "wavefront-small-waves", "wavefront-two-level"])
def test_tuning_does_not_change_results(scene_ctx, tuning):
    s, c = scene_ctx
    tuning = dict(tuning)
    width = tuning.pop("bvh_width", 0)  # a BVH layout of its own: built for this case, rebuilt after
    if width:
        c.build(width=width)
    try:
        c.set_tuning()
        ref, st0 = _film(c, s)
        c.set_tuning(**tuning)
        out, st1 = _film(c, s)
    finally:
        c.set_tuning()
        if width:
            c.build()
    assert np.array_equal(out, ref)
    assert st1.traced == st0.traced
    if tuning.get("trace_mode") == 3:  # one launch per chunk for all of its waves
        assert st1.kernels < st0.kernels
        if "queue_capacity" not in tuning:
            assert st1.waves == st0.waves
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


def test_wavefront_batch_matches_single_renders():
    """trace_mode 3 over a batch of contexts: each film equals the context's own default render."""
    from axomae_b200 import native, scenes
    specs = [(scenes.mixed_scene(12000, 48, 40, seed=3), 48, 40, 16, 6),
             (scenes.spheres_scene(40, 24, n_spheres=7, seed=8), 40, 24, 8, 5),
             (scenes.mixed_scene(6000, 33, 17, seed=4), 33, 17, 4, 3)]
    ctxs = []
    try:
        frames, refs = [], []
        for s, W, H, spp, depth in specs:
            c = native.Context(0)
            ctxs.append(c)
            c.upload(s)
            c.build()
            fr = native.make_frame(s, W, H, spp, depth)
            ref = np.zeros((H, W, 4), np.float32)
            c.render(fr, film_host=ref)
            frames.append(fr)
            refs.append(ref)
            c.set_tuning(trace_mode=3)
        outs = [np.zeros_like(r) for r in refs]
        st = native.render_batch(ctxs, frames, films_host=outs)
        for o, r in zip(outs, refs):
            assert np.array_equal(o, r)
        assert st.traced > 0
    finally:
        for c in ctxs:
            c.close()


def test_wavefront_barrier_wait_limit_fails_the_render(scene_ctx):
    """A grid-barrier wait longer than wait_limit_us ends the persistent launch: the render fails with
    RENDERER_EXCEPTION naming the limit, and the context renders correctly afterwards.  With a limit of
    1 us some block always waits longer for the others (a wave's trace phase alone takes far longer)."""
    from axomae_b200 import native
    s, c = scene_ctx
    c.set_tuning()
    ref, _ = _film(c, s)
    c.set_tuning(trace_mode=3, wait_limit_us=1, queue_capacity=65536)
    try:
        with pytest.raises(native.NovaError) as e:
            _film(c, s, spp=64)
        assert e.value.status == 16 and "grid barrier" in str(e.value)
    finally:
        c.set_tuning()
    again, _ = _film(c, s)
    assert np.array_equal(again, ref)
    c.set_tuning(trace_mode=3)
    try:
        out, _ = _film(c, s)
    finally:
        c.set_tuning()
    assert np.array_equal(out, ref)


def test_wavefront_cancel_stops_the_launch():
    """nova_b200_cancel during a persistent launch: the kernel sees the mapped flag at its next wave end,
    returns, and the render fails with RENDERER_EXCEPTION within a short time."""
    import threading
    import time
    import torch
    from axomae_b200 import native, scenes
    s = scenes.spheres_scene(64, 64, n_spheres=8, seed=1)
    c = native.Context(0)
    try:
        c.upload(s)
        c.build()
        c.set_tuning(trace_mode=3)
        film = torch.zeros(1024 * 1024 * 4, device="cuda")
        long_frame = native.make_frame(s, 1024, 1024, 2048, 8)  # 2^31 paths: seconds of work
        result = {}

        def run():
            try:
                c.render(long_frame, film_device_ptr=film.data_ptr())
                result["done"] = True
            except native.NovaError as e:
                result["error"] = e

        t = threading.Thread(target=run)
        t.start()
        time.sleep(0.3)
        t0 = time.perf_counter()
        c.cancel()
        t.join(timeout=60)
        stopped = time.perf_counter() - t0
        assert not t.is_alive()
        assert "error" in result, "the render finished before the cancel"
        assert result["error"].status == 16 and "cancel" in str(result["error"])
        assert stopped < 2.0
        small = native.make_frame(s, 64, 64, 4, 4)
        a = np.zeros((64, 64, 4), np.float32)
        c.render(small, film_host=a)
        c.set_tuning()
        b = np.zeros((64, 64, 4), np.float32)
        c.render(small, film_host=b)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    finally:
        c.close()

"""Parity of the CUDA path (through the C ABI) with the CPU oracle on seeded scenes.

Bars: Sobol/Owen values bit-exact; closest-hit primitive identical
and distance within 2 ulp for primary rays except exact ties; rendered images within a per-pixel
relative RMSE of 1e-3 (relative error (gpu - ref) / max(ref, 1e-3), RGB)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
REL_RMSE_TOL = 1e-3


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return torch


@pytest.fixture(scope="module")
def ctx(torch_cuda):
    from axomae_b200 import native
    c = native.Context(0)
    yield c
    c.close()


def rel_rmse(gpu, ref):
    d = (gpu[..., :3].astype(np.float64) - ref[..., :3]) / np.maximum(ref[..., :3], 1e-3)
    return float(np.sqrt(np.mean(d * d)))


def ulp_diff(a, b):
    ai = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    bi = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    ai = np.where(ai < 0, -(ai & 0x7FFFFFFF), ai)
    bi = np.where(bi < 0, -(bi & 0x7FFFFFFF), bi)
    return np.abs(ai - bi)


def test_sobol_bit_exact(ctx, oracle, torch_cuda):
    torch = torch_cuda
    g = np.load(os.path.join(GOLDEN, "sobol_samples.npz"))
    rng = np.random.default_rng(1)
    for seed in (0, 0xDEADBEEF, 12345):
        idx = np.concatenate([g["index"], rng.integers(0, 2**32, 20000, dtype=np.uint64).astype(np.uint32)])
        dim = np.concatenate([g["dim"], rng.integers(0, 255, 20000).astype(np.uint32)])
        ti = torch.from_numpy(idx.view(np.int32)).cuda()
        td = torch.from_numpy(dim.view(np.int32)).cuda()
        out = torch.empty(idx.size, dtype=torch.float32, device="cuda")
        ctx.sobol(ti.data_ptr(), td.data_ptr(), idx.size, seed, out.data_ptr())
        dev = out.cpu().numpy()
        ref = oracle.sobol_samples(idx, dim, seed)
        assert np.array_equal(dev.view(np.uint32), ref.view(np.uint32))
        m = g["seed"] == seed
        if m.any():
            assert np.array_equal(dev[: g["index"].size][m].view(np.uint32), g["bits"][m])


def _trace(ctx, torch, o, d):
    n = o.shape[0]
    to = torch.from_numpy(np.ascontiguousarray(o, np.float32)).cuda()
    td = torch.from_numpy(np.ascontiguousarray(d, np.float32)).cuda()
    prim = torch.empty(n, dtype=torch.int32, device="cuda")
    t, u, v = (torch.empty(n, dtype=torch.float32, device="cuda") for _ in range(3))
    ctx.trace(to.data_ptr(), td.data_ptr(), n, prim.data_ptr(), t.data_ptr(), u.data_ptr(), v.data_ptr())
    return prim.cpu().numpy(), t.cpu().numpy(), u.cpu().numpy(), v.cpu().numpy()


def _check_hits(ctx, torch, osc, o, d, max_mismatch_frac):
    p_ref, t_ref, u_ref, v_ref, _ = osc.trace(o, d)
    p_dev, t_dev, u_dev, v_dev = _trace(ctx, torch, o, d)
    same = p_ref == p_dev
    # a differing primitive is acceptable only on an exact distance tie
    diff = ~same
    tie = diff & (p_ref >= 0) & (p_dev >= 0) & (t_ref == t_dev)
    bad = diff & ~tie
    assert bad.mean() <= max_mismatch_frac, "primitive mismatches: %d of %d" % (bad.sum(), len(bad))
    hit = same & (p_ref >= 0)
    assert np.all(ulp_diff(t_dev[hit], t_ref[hit]) <= 2)
    return hit.sum(), bad.sum()


@pytest.fixture(scope="module")
def spheres_scene(oracle):
    from axomae_b200 import scenes
    s = scenes.spheres_scene(96, 96)
    return s, oracle.OracleScene(s)


@pytest.fixture(params=[8, 2], ids=["bvh8", "bvh2"])
def spheres(ctx, spheres_scene, request):
    s, osc = spheres_scene
    ctx.upload(s)
    ctx.build(width=request.param)
    return s, osc


def test_primary_ray_hits(ctx, oracle, spheres, torch_cuda):
    s, osc = spheres
    W = H = 96
    opt = oracle.options(W, H, 4, 5)
    ys, xs = np.mgrid[0:H, 0:W]
    px, py = xs.reshape(-1), ys.reshape(-1)
    for sample in range(4):
        o, d = osc.camera_rays(opt, px, py, np.full(px.size, sample))
        nhit, nbad = _check_hits(ctx, torch_cuda, osc, o, d, 0.0)
        assert nhit > 0.3 * px.size


def test_random_ray_hits(ctx, oracle, spheres, torch_cuda):
    s, osc = spheres
    rng = np.random.default_rng(7)
    n = 50000
    o = rng.uniform([-10, 0.05, -10], [10, 3, 10], (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    _check_hits(ctx, torch_cuda, osc, o, d.astype(np.float32), 1e-4)


def _render(ctx, scene, W, H, spp, depth, rr=-1, seed=0):
    from axomae_b200 import native
    film = np.zeros((H, W, 4), np.float32)
    fr = native.make_frame(scene, W, H, spp, depth, seed=seed, rr_start=rr)
    stats = ctx.render(fr, film_host=film)
    return film, stats


def test_render_spheres_matches_oracle(ctx, oracle, spheres):
    s, osc = spheres
    W = H = 96
    film, stats = _render(ctx, s, W, H, 16, 5)
    ref, rst = osc.render(oracle.options(W, H, 16, 5, threads=0))
    assert np.isfinite(film).all()
    err = rel_rmse(film, ref)
    assert err <= REL_RMSE_TOL, err
    assert stats.paths == W * H * 16


def test_render_mixed_materials_matches_oracle(ctx, oracle):
    from axomae_b200 import scenes
    s = scenes.mixed_scene(20000, 64, 64, seed=3)
    ctx.upload(s)
    ctx.build()
    film, _ = _render(ctx, s, 64, 64, 16, 6)
    ref, _ = oracle.OracleScene(s).render(oracle.options(64, 64, 16, 6))
    err = rel_rmse(film, ref)
    assert err <= REL_RMSE_TOL, err


def test_render_heightfield_rr_matches_oracle(ctx, oracle):
    from axomae_b200 import scenes
    s = scenes.heightfield_scene(n=64, width=80, height=45, env_w=128, env_h=64, seed=5)
    ctx.upload(s)
    ctx.build()
    film, _ = _render(ctx, s, 80, 45, 16, 8, rr=3)
    ref, _ = oracle.OracleScene(s).render(oracle.options(80, 45, 16, 8, rr_start=3))
    err = rel_rmse(film, ref)
    assert err <= REL_RMSE_TOL, err


def test_progressive_sample_ranges_equal_one_shot(ctx, oracle):
    """Frames of sample ranges accumulated on the device film equal one call over all samples
    (running mean of writeFramebuffer, api/engine.cpp:351-363)."""
    from axomae_b200 import native, scenes
    s = scenes.spheres_scene(48, 48, n_spheres=8)
    ctx.upload(s)
    ctx.build()
    one = np.zeros((48, 48, 4), np.float32)
    ctx.render(native.make_frame(s, 48, 48, 8, 4), film_host=one)
    prog = np.zeros_like(one)
    for b in range(0, 8, 2):
        ctx.render(native.make_frame(s, 48, 48, 8, 4, sample_begin=b, sample_count=2, reset=int(b == 0)),
                   film_host=prog)
    np.testing.assert_allclose(prog[..., :3], one[..., :3], rtol=2e-6, atol=1e-7)


def test_bake_matches_oracle(ctx, oracle, torch_cuda):
    torch = torch_cuda
    rng = np.random.default_rng(11)
    src = np.concatenate([rng.lognormal(0, 1, (64, 128, 3)), np.ones((64, 128, 1))], -1).astype(np.float32)
    ref = oracle.bake_irradiance(src, 32, 16, 64)
    ts = torch.from_numpy(src).cuda()
    out = torch.zeros((16, 32, 4), dtype=torch.float32, device="cuda")
    ctx.bake_irradiance(ts.data_ptr(), 128, 64, 4, 32, 16, 64, out.data_ptr())
    dev = out.cpu().numpy()
    np.testing.assert_allclose(dev[..., :3], ref[..., :3], rtol=1e-4, atol=1e-6)


def test_error_paths(ctx):
    from axomae_b200 import native, scenes
    s = scenes.spheres_scene(16, 16, n_spheres=2)
    ctx.upload(s)
    with pytest.raises(native.NovaError) as e:
        ctx.render(native.make_frame(s, 16, 16, 1, 2))
    assert e.value.status == 9  # SCENE_NOT_PROCESSED
    ctx.build()
    with pytest.raises(native.NovaError) as e:
        ctx.render(native.make_frame(s, 16, 16, 4, 2, sample_begin=3, sample_count=2))
    assert e.value.status == 15  # INVALID_ARGUMENT
    with pytest.raises(native.NovaError) as e:
        ctx.render(native.make_frame(s, 16, 16, 4, 99))
    assert e.value.status == 15
    bad = dict(s)
    bad["envmap"] = 0  # an 8-bit texture cannot be the environment
    with pytest.raises(native.NovaError) as e:
        ctx.upload(bad)
    assert e.value.status == 4  # INVALID_SCENE_TYPE


def test_batch_calls_reject_bad_arguments(torch_cuda):
    """The batch entry points check their arguments before any work: an empty batch, a null scene or
    frame array, a frame with an invalid sample range, and two jobs on one context fail with
    INVALID_ARGUMENT, and the contexts stay usable."""
    import ctypes as C
    from axomae_b200 import native, scenes
    s = scenes.spheres_scene(16, 12, n_spheres=2, seed=9)
    a, b = native.Context(0), native.Context(0)
    try:
        L = native.lib()
        hs = (C.c_void_p * 2)(a.h, b.h)
        opts = native.BvhOptions(0, 0, 0, 0)
        assert L.nova_b200_upload_build_batch(hs, None, 2, C.byref(opts)) == 15
        assert L.nova_b200_upload_build_render_batch(hs, None, None, 2, None, None, None, None) == 15
        good = native.make_frame(s, 16, 12, 4, 3)
        bad = native.make_frame(s, 16, 12, 4, 3, sample_begin=3, sample_count=2)
        with pytest.raises(native.NovaError) as e:
            native.upload_build_render_batch([a, b], [s, s], [good, bad])
        assert e.value.status == 15
        with pytest.raises(native.NovaError) as e:
            native.upload_build_render_batch([a, a], [s, s], [good, good])
        assert e.value.status == 15
        native.upload_build_batch([a, b], [s, s])
        fa, fb = np.zeros((12, 16, 4), np.float32), np.zeros((12, 16, 4), np.float32)
        native.render_batch([a, b], [good, good], films_host=[fa, fb])
        assert np.array_equal(fa, fb) and np.isfinite(fa).all()
    finally:
        a.close()
        b.close()


def test_upload_checks_indices_and_degenerate_triangles(ctx, oracle, torch_cuda):
    """The per-triangle scene tables are built on the device: an index past its mesh's vertices is
    rejected (INVALID_ARGUMENT), a scene of only degenerate triangles too (INVALID_SCENE_TYPE, as
    Triangle.h:127-132 makes them unhittable), and the context stays usable; triangles with a
    repeated index are left out of the BVH, so hits agree with the oracle."""
    import copy
    from axomae_b200 import native, scenes
    s = scenes.spheres_scene(48, 48, n_spheres=6, seed=4)
    bad = copy.deepcopy(s)
    idx = np.array(bad["meshes"][1]["indices"], np.uint32).reshape(-1)
    idx[7] = len(np.asarray(bad["meshes"][1]["vertices"]).reshape(-1, 3))
    bad["meshes"][1]["indices"] = idx.reshape(np.shape(s["meshes"][1]["indices"]))
    with pytest.raises(native.NovaError) as e:
        ctx.upload(bad)
    assert e.value.status == 15
    flat = copy.deepcopy(s)
    for m in flat["meshes"]:
        ix = np.array(m["indices"], np.uint32).reshape(-1, 3)
        ix[:, 1] = ix[:, 0]
        m["indices"] = ix.reshape(np.shape(m["indices"]))
    with pytest.raises(native.NovaError) as e:
        ctx.upload(flat)
    assert e.value.status == 4
    half = copy.deepcopy(s)
    rng = np.random.default_rng(3)
    for m in half["meshes"]:
        ix = np.array(m["indices"], np.uint32).reshape(-1, 3)
        sel = rng.random(len(ix)) < 0.3
        ix[sel, 2] = ix[sel, 1]
        m["indices"] = ix.reshape(np.shape(m["indices"]))
    ctx.upload(half)
    ctx.build()
    osc = oracle.OracleScene(half)
    assert ctx.info()["triangles"] == sum(np.size(half["meshes"][x["mesh"]]["indices"]) // 3 for x in half["instances"])
    o = rng.uniform([-10, 0.05, -10], [10, 3, 10], (20000, 3)).astype(np.float32)
    d = rng.normal(size=(20000, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    _check_hits(ctx, torch_cuda, osc, o, d, 1e-4)
    film, _ = _render(ctx, half, 48, 48, 8, 4)
    ref, _ = osc.render(oracle.options(48, 48, 8, 4))
    assert rel_rmse(film, ref) <= REL_RMSE_TOL


def test_cancel_stops_a_long_render(torch_cuda):
    """nova_b200_cancel from another thread stops a long render within a few wave groups with
    RENDERER_EXCEPTION, and the context renders correctly afterwards."""
    import threading
    import time
    from axomae_b200 import native, scenes
    torch = torch_cuda
    s = scenes.spheres_scene(64, 64, n_spheres=8, seed=1)
    c = native.Context(0)
    try:
        c.upload(s)
        c.build()
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
        fresh = native.Context(0)
        try:
            fresh.upload(s)
            fresh.build()
            b = np.zeros((64, 64, 4), np.float32)
            fresh.render(small, film_host=b)
        finally:
            fresh.close()
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    finally:
        c.close()


def test_upload_from_pinned_memory_equals_pageable(ctx, torch_cuda):
    """Scene arrays in pinned host memory are read by the device's gather kernel, pageable ones go
    through the staging buffer: both uploads give the same BVH and the same image bit for bit."""
    import bench
    from axomae_b200 import native, scenes
    s = scenes.mixed_scene(20000, 40, 32, seed=5)
    pinned = native.prepare_scene(bench.pin_scene(s))
    other = native.Context(0)
    try:
        ctx.upload(s)
        ctx.build()
        other.upload(pinned)
        other.build()
        tree = lambda c: {k: v for k, v in c.info().items() if k != "device_bytes"}  # render buffers differ
        assert tree(ctx) == tree(other)
        fr = native.make_frame(s, 40, 32, 4, 4)
        a, b = np.zeros((32, 40, 4), np.float32), np.zeros((32, 40, 4), np.float32)
        ctx.render(fr, film_host=a)
        other.render(fr, film_host=b)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    finally:
        other.close()


def test_bvh_independent_of_subtree_threshold(ctx, torch_cuda):
    """Nodes above the subtree threshold are split by the level kernels, smaller ones inside one CTA
    (binned SAH, stable partition) and those of <= 32 primitives by warp lane segments (exact sweep).
    The level kernels and the CTA path take the same binned decisions, so moving the threshold
    gives the same tree: the same node and leaf counts, node visits per ray and film bit for bit."""
    from axomae_b200 import native, scenes
    s = scenes.mixed_scene(60000, 40, 32, seed=9)
    fr = native.make_frame(s, 40, 32, 4, 6)
    ctx.upload(s)
    out = []
    for small in (64, 256, 4096):
        ctx.build(small_subtree=small)
        info = {k: v for k, v in ctx.info().items() if k != "device_bytes"}
        film = np.zeros((32, 40, 4), np.float32)
        ctx.render(fr, film_host=film)
        ctx.set_tuning(trace_mode=2)
        st = ctx.render(fr, film_host=np.zeros_like(film))
        ctx.set_tuning()
        out.append((info, film, st.node_visits, st.tri_tests))
    for info, film, nv, tt in out[1:]:
        assert info == out[0][0]
        assert np.array_equal(film.view(np.uint32), out[0][1].view(np.uint32))
        assert (nv, tt) == (out[0][2], out[0][3])


def test_batch_equals_individual_renders(torch_cuda):
    """nova_b200_render_batch: frames of different scenes, sizes, sample counts and depths rendered
    as one wavefront equal the same frames rendered one by one, bit for bit."""
    from axomae_b200 import native, scenes
    specs = [(scenes.spheres_scene(40, 30, n_spheres=6, seed=1), 40, 30, 4, 3, -1),
             (scenes.mixed_scene(8000, 24, 16, seed=2), 24, 16, 8, 6, 2),
             (scenes.heightfield_scene(n=32, width=33, height=17, env_w=64, env_h=32, seed=3), 33, 17, 1, 8, 3)]
    ctxs, frames, refs = [], [], []
    try:
        for s, W, H, spp, depth, rr in specs:
            c = native.Context(0)
            ctxs.append(c)
            c.upload(s)
            c.build()
            fr = native.make_frame(s, W, H, spp, depth, rr_start=rr)
            frames.append(fr)
            ref = np.zeros((H, W, 4), np.float32)
            c.render(fr, film_host=ref)
            refs.append(ref)
        outs = [np.zeros_like(r) for r in refs]
        st = native.render_batch(ctxs, frames, films_host=outs)
        for o, r in zip(outs, refs):
            assert np.array_equal(o, r)
        assert st.paths == sum(W * H * spp for _, W, H, spp, _, _ in specs)
    finally:
        for c in ctxs:
            c.close()


def test_batch_of_several_chunks_copies_every_film(torch_cuda):
    """A batch of 110 frames spans two chunks (104 jobs per chunk): the films of the first chunk's
    frames go out while the second chunk renders (pinned host and device films), pageable host films
    after the render; every film equals the frame rendered alone, bit for bit."""
    from axomae_b200 import native, scenes
    torch = torch_cuda
    n, W, H = 110, 16, 12
    specs = [scenes.spheres_scene(W, H, n_spheres=2 + k % 4, seed=100 + k) for k in range(n)]
    ctxs = [native.Context(0) for _ in range(n)]
    try:
        native.upload_build_batch(ctxs, specs)
        frames = [native.make_frame(s, W, H, 4, 4) for s in specs]
        refs = []
        for c, fr in zip(ctxs, frames):
            ref = np.zeros((H, W, 4), np.float32)
            c.render(fr, film_host=ref)
            refs.append(ref)
        pinned = [torch.zeros((H, W, 4), dtype=torch.float32).pin_memory() for _ in range(n)]
        device = [torch.zeros((H, W, 4), dtype=torch.float32, device="cuda") for _ in range(n)]
        pageable = [np.zeros((H, W, 4), np.float32) for _ in range(n)]
        hosts = [pinned[j].numpy() if j % 3 == 0 else (pageable[j] if j % 3 == 2 else None) for j in range(n)]
        devs = [device[j].data_ptr() if j % 3 == 1 else None for j in range(n)]
        st = native.render_batch(ctxs, frames, films_host=hosts, films_device=devs)
        assert st.paths == n * W * H * 4
        for j in range(n):
            got = hosts[j] if j % 3 != 1 else device[j].cpu().numpy()
            assert np.array_equal(got, refs[j]), j
    finally:
        for c in ctxs:
            c.close()


def test_pipelined_upload_build_render_equals_separate_calls(torch_cuda):
    """nova_b200_upload_build_render_batch (uploads and builds on host threads while the chunks whose
    scenes are ready render) gives the films of the three separate batch calls, bit for bit, over a
    110-frame batch of two chunks; a scene that fails to upload fails the call without a hang, and
    the contexts render normally afterwards."""
    from axomae_b200 import native, scenes
    torch = torch_cuda
    n, W, H = 110, 16, 12
    specs = [scenes.spheres_scene(W, H, n_spheres=2 + k % 4, seed=300 + k) for k in range(n)]
    frames = [native.make_frame(s, W, H, 4, 4) for s in specs]
    a = [native.Context(0) for _ in range(n)]
    b = [native.Context(0) for _ in range(n)]
    try:
        native.upload_batch(a, specs)
        native.build_batch(a)
        refs = [np.zeros((H, W, 4), np.float32) for _ in range(n)]
        native.render_batch(a, frames, films_host=refs)
        pinned = [torch.zeros((H, W, 4), dtype=torch.float32).pin_memory() for _ in range(n)]
        outs = [p.numpy() for p in pinned]
        st = native.upload_build_render_batch(b, specs, frames, films_host=outs)
        assert st.paths == n * W * H * 4
        for ca, cb in zip(a, b):
            assert ca.info() == cb.info()
        for o, r in zip(outs, refs):
            assert np.array_equal(o, r)
        bad = list(specs)
        broken = dict(specs[57])
        broken["instances"] = [dict(x) for x in specs[57]["instances"]]
        broken["instances"][0]["mesh"] = len(broken["meshes"]) + 5
        bad[57] = broken
        with pytest.raises(native.NovaError) as e:
            native.upload_build_render_batch(b, bad, frames, films_host=outs)
        assert e.value.status == 15 and "missing mesh" in str(e.value)
        again = np.zeros((H, W, 4), np.float32)
        b[3].render(frames[3], film_host=again)
        assert np.array_equal(again, refs[3])
    finally:
        for c in a + b:
            c.close()


def test_scatter_bit_exact(ctx, oracle, torch_cuda):
    """nova_b200_scatter (hit record + principled scatter + spawn) equals the oracle bit for bit on
    the hits of oracle paths through a mixed Lambert / GGX conductor / GGX dielectric scene."""
    from axomae_b200 import scenes
    torch = torch_cuda
    s = scenes.mixed_scene(30000, 48, 48, seed=11)
    ctx.upload(s)
    ctx.build()
    osc = oracle.OracleScene(s)
    W = H = 48
    spp, depth = 8, 8
    opt = oracle.options(W, H, spp, depth)
    rng = np.random.default_rng(5)
    rows, idx, bnc = [], [], []
    for _ in range(1500):
        x, y, smp = int(rng.integers(W)), int(rng.integers(H)), int(rng.integers(spp))
        segs, _ = osc.sample_path(opt, x, y, smp)
        for b, r in enumerate(segs):
            if np.float32(r[6]).view(np.int32) >= 0 and b <= depth:
                rows.append(r)
                idx.append((x * H + y) * spp + smp)
                bnc.append(b)
    R = np.asarray(rows, np.float32)
    n = R.shape[0]
    prim = R[:, 6].copy().view(np.int32)
    index = np.asarray(idx, np.uint32)
    bounce = np.asarray(bnc, np.int32)
    ref = osc.scatter(R[:, :3], R[:, 3:6], prim, R[:, 7], R[:, 8], R[:, 9], index, bounce)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    ins = [T(R[:, :3]), T(R[:, 3:6]), T(prim), T(R[:, 7]), T(R[:, 8]), T(R[:, 9]), T(index.view(np.int32)), T(bounce)]
    outs = [torch.zeros((n, 3), dtype=torch.float32, device="cuda") for _ in range(4)]
    valid = torch.zeros(n, dtype=torch.int32, device="cuda")
    ctx.scatter(n, *[a.data_ptr() for a in ins], 0, *[a.data_ptr() for a in outs], valid.data_ptr())
    dev = [a.cpu().numpy() for a in outs]
    v_dev = valid.cpu().numpy()
    assert np.array_equal(v_dev, ref[4])
    ok = v_dev == 1
    assert ok.sum() > 0.8 * n
    for a, b in zip(dev, ref[:4]):
        assert np.array_equal(a[ok].view(np.uint32), b[ok].view(np.uint32))


def test_converged_4096spp(ctx, oracle):
    """Converged image of the 64-sphere scene at 4096 spp: per-pixel relative RMSE <= 1e-3."""
    from axomae_b200 import scenes
    W = H = 24
    s = scenes.spheres_scene(W, H)
    ctx.upload(s)
    ctx.build()
    film, st = _render(ctx, s, W, H, 4096, 5)
    ref, _ = oracle.OracleScene(s).render(oracle.options(W, H, 4096, 5))
    err = rel_rmse(film, ref)
    assert err <= REL_RMSE_TOL, err
    assert st.paths == W * H * 4096


@pytest.fixture(scope="module")
def batch_jobs():
    from axomae_b200 import scenes
    return scenes.batch_jobs(32, seed=0)


@pytest.mark.parametrize("job", [0, 7, 12, 30])
def test_batch_workload_scene_matches_oracle(job, ctx, oracle, batch_jobs):
    """Scenes of the 32-job batched workload (dielectric-heavy, depth up to 12) at 48 x 48 with the
    job's spp and depth, against the oracle."""
    j = batch_jobs[job]
    W = H = 48
    ctx.upload(j["scene"])
    ctx.build()
    film, _ = _render(ctx, j["scene"], W, H, j["spp"], j["depth"])
    ref, _ = oracle.OracleScene(j["scene"]).render(oracle.options(W, H, j["spp"], j["depth"]))
    err = rel_rmse(film, ref)
    assert err <= REL_RMSE_TOL, err


@pytest.mark.parametrize("width", [2, 8, 1], ids=["bvh2", "bvh8", "two_level"])
def test_instanced_scene_matches_oracle(ctx, oracle, torch_cuda, width):
    """Seeded meshes placed many times with random rigid transforms: rays are brought into each
    instance's object space (Triangle.h:150-153) exactly as the reference does, with the flat BVHs
    over every instanced triangle and with the two-level one (a BVH per mesh under a BVH over the
    instances, as the reference's Embree scene keeps them, embree.cpp:236-254)."""
    from axomae_b200 import scenes
    s = scenes.instanced_scene(n_meshes=3, n_instances=40, tris_per_mesh=1500, width=64, height=48, seed=8,
                               box_size=20.0, env_w=64, env_h=32)
    ctx.upload(s)
    ctx.build(width=width)
    film, _ = _render(ctx, s, 64, 48, 8, 8)
    osc = oracle.OracleScene(s)
    ref, _ = osc.render(oracle.options(64, 48, 8, 8))
    assert rel_rmse(film, ref) <= REL_RMSE_TOL
    rng = np.random.default_rng(3)
    n = 40000
    o = rng.uniform(-12, 12, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    _check_hits(ctx, torch_cuda, osc, o, d.astype(np.float32), 1e-4)


def test_batch_upload_and_build_equal_single_calls(torch_cuda):
    """nova_b200_upload_scene_batch / nova_b200_build_bvh_batch and nova_b200_upload_build_batch
    (contexts concurrently) give the same BVHs and images as one call per context."""
    from axomae_b200 import native, scenes
    specs = [scenes.mixed_scene(6000 + 3000 * k, 24, 20, seed=20 + k) for k in range(5)]
    a = [native.Context(0) for _ in specs]
    b = [native.Context(0) for _ in specs]
    f = [native.Context(0) for _ in specs]
    try:
        native.upload_batch(a, specs)
        native.build_batch(a)
        native.upload_build_batch(f, specs)
        for c, s in zip(b, specs):
            c.upload(s)
            c.build()
        for ca, cb, cf, s in zip(a, b, f, specs):
            assert ca.info() == cb.info() == cf.info()
            fa, fb, ff = (np.zeros((20, 24, 4), np.float32) for _ in range(3))
            fr = native.make_frame(s, 24, 20, 4, 5)
            ca.render(fr, film_host=fa)
            cb.render(fr, film_host=fb)
            cf.render(fr, film_host=ff)
            assert np.array_equal(fa, fb) and np.array_equal(ff, fb)
        with pytest.raises(native.NovaError):
            native.build_batch([a[0], a[0]])
        with pytest.raises(native.NovaError):
            native.upload_build_batch([f[0], f[0]], specs[:2])
    finally:
        for c in a + b + f:
            c.close()


@pytest.fixture(scope="module")
def emissive_scene():
    """Mixed scene where a quarter of the materials emit (u8 emissive texture) and a third carry a
    seeded bumpy normal map."""
    from axomae_b200 import scenes
    s = scenes.mixed_scene(15000, 56, 40, seed=31)
    rng = np.random.default_rng(31)
    tex = list(s["textures"])
    mats = [dict(m) for m in s["materials"]]
    for i, m in enumerate(mats):
        if i % 4 == 1:
            tex.append(scenes.solid_u8(rng.uniform(0.2, 3.0, 3).clip(0, 1)))
            m["emissive"] = len(tex) - 1
        if i % 3 == 2:
            nm = np.concatenate([rng.integers(90, 166, (8, 8, 2)), rng.integers(200, 256, (8, 8, 1)),
                                 np.full((8, 8, 1), 255)], -1).astype(np.uint8)
            tex.append(scenes.u8_texture(nm))
            m["normalmap"] = len(tex) - 1
    return dict(s, textures=tex, materials=mats)


def test_render_emissive_normal_mapped_matches_oracle(ctx, oracle, emissive_scene):
    s = emissive_scene
    ctx.upload(s)
    ctx.build()
    film, _ = _render(ctx, s, 56, 40, 16, 6)
    ref, _ = oracle.OracleScene(s).render(oracle.options(56, 40, 16, 6))
    assert rel_rmse(film, ref) <= REL_RMSE_TOL


@pytest.mark.parametrize("kind,name", [(1, "normal"), (2, "depth"), (4, "emissive")])
@pytest.mark.parametrize("vinv", [0, 1])
def test_aov_matches_oracle(ctx, oracle, emissive_scene, kind, name, vinv):
    """Normal, depth and emissive AOV integrators, value for value.  The frame is odd-sized: the AOV
    camera rays carry no jitter, and a ray through the exact centre line of an even frame can have
    a zero direction component; where its origin lies on a box plane, the reference's slab test
    divides 0 by 0 and culls the box (BoundingBox.cpp:150-160), which the device's test does not."""
    from axomae_b200 import native
    s = emissive_scene
    ctx.upload(s)
    ctx.build()
    W, H = 57, 41
    fr = native.make_frame(s, W, H, 1, 4, vertical_invert=vinv)
    out = np.zeros((H, W, 4), np.float32)
    ctx.render_aov(fr, kind, 0.1, 1000.0, film_host=out)
    opt = oracle.options(W, H, 1, 4, vertical_invert=vinv)
    ref = oracle.OracleScene(s).render_aov(opt, kind, 0.1, 1000.0)
    hit = ref[..., 3] != 0 if kind != 2 else ref[..., 0] != 1000.0
    assert hit.mean() > 0.2
    # identical except where the closest hit is a tie between two triangles
    same = np.all(out == ref, axis=-1)
    assert same.mean() >= 0.999, (name, same.mean())
    if kind == 4:
        assert (out[..., :3].max(-1) > 0).any()


def test_device_status_counts_nonfinite_radiance(ctx, oracle, torch_cuda):
    """The device status word, from a host-made bad input: every 7th triangle gets a NaN albedo (per-
    triangle albedo of the differentiable parameters).  Paths through those triangles carry NaN
    weights; the device writes their radiance as 0 (the reference's DENAN, Integrator.cpp:92), counts
    them in the stats' `nonfinite`, and the film stays finite and equal to the oracle's, which applies
    DENAN at every level.  A clean render reports zero, and no index error either way."""
    from axomae_b200 import native, scenes
    W = H = 48
    s = scenes.spheres_scene(W, H, n_spheres=8, seed=2)
    ctx.upload(s)
    ctx.build()
    ntri = ctx.info()["triangles"]
    nmat = len(s["materials"])
    alb = np.full((ntri, 3), 0.5, np.float32)
    rough = np.full(nmat, 0.3, np.float32)
    fr = native.make_frame(s, W, H, 8, 4)
    osc = oracle.OracleScene(s)
    results = {}
    for name in ("clean", "nan"):
        a = alb.copy()
        if name == "nan":
            a[::7] = np.nan
        ta, tr = torch_cuda.from_numpy(a).cuda(), torch_cuda.from_numpy(rough).cuda()
        ctx.set_diff_params(ta.data_ptr(), tr.data_ptr())
        film = np.zeros((H, W, 4), np.float32)
        try:
            st = ctx.render(fr, film_host=film)
        finally:
            ctx.set_diff_params(None, None)
        osc.set_diff_params(a, rough)
        ref, _ = osc.render(oracle.options(W, H, 8, 4))
        results[name] = (st, film, ref)
    st, film, ref = results["clean"]
    assert st.nonfinite == 0 and st.bad_index == 0
    st, film, ref = results["nan"]
    assert st.bad_index == 0
    assert st.nonfinite > 100, st.nonfinite
    assert np.isfinite(film).all()
    assert rel_rmse(film, ref) <= REL_RMSE_TOL
    assert film[..., :3].mean() < results["clean"][1][..., :3].mean()  # the zeroed paths darken the image


@pytest.mark.parametrize("channels", [4, 3])
def test_bake_texunit_matches_oracle(ctx, oracle, torch_cuda, channels):
    """The reference's CUDA bake (the --gpu path, CubemapProcessing.cu:129-175): hash seeded with the
    output texel, exact acos / atan2f, hardware bilinear filtering with wrap addressing.  The oracle
    restates the texture unit's filter from the CUDA programming guide (8-bit fractional weights) with
    correctly rounded trigonometry, so the two agree within rel. RMSE 1e-3, not bit for bit; an RGB
    source bakes as the same map with alpha 1; the output alpha is 1."""
    torch = torch_cuda
    rng = np.random.default_rng(13)
    src = np.concatenate([rng.lognormal(0, 1.5, (256, 512, 3)), np.ones((256, 512, 1))], -1).astype(np.float32)
    src = np.ascontiguousarray(src[..., :channels])
    ts = torch.from_numpy(src).cuda()
    for ow, oh in ((64, 64), (128, 32)):
        out = torch.full((oh, ow, 4), -1.0, dtype=torch.float32, device="cuda")
        ctx.bake_irradiance_texunit(ts.data_ptr(), 512, 256, channels, ow, oh, 128, out.data_ptr())
        dev = out.cpu().numpy()
        ref = oracle.bake_irradiance_texunit(src, ow, oh, 128)
        assert (dev[..., 3] == 1.0).all()
        assert rel_rmse(dev, ref) <= 1e-3, rel_rmse(dev, ref)
        cpu_path = oracle.bake_irradiance(np.concatenate([src[..., :3], np.ones_like(src[..., :1])], -1), ow, oh, 128)
        assert rel_rmse(dev, cpu_path) > 1e-2  # a different estimator from the CPU path's, as in the reference


def test_two_level_bvh_edge_cases(ctx, oracle, torch_cuda):
    """The two-level BVH with one mesh under many instances (shared bottom level), an identity
    instance (the world ray kept bit for bit), an unused mesh, and a mesh whose triangles are all
    degenerate (never hit, Triangle.h:127-132): hits equal the oracle's except exact ties, images
    within 1e-3, and the same closest primitives as the flat BVH."""
    from axomae_b200 import scenes
    s = scenes.instanced_scene(n_meshes=3, n_instances=30, tris_per_mesh=800, width=48, height=40, seed=12,
                               box_size=16.0, env_w=64, env_h=32)
    meshes = list(s["meshes"])
    deg = dict(meshes[0])
    deg["indices"] = np.repeat(np.asarray(meshes[0]["indices"]).reshape(-1, 3)[:, :1], 3, axis=1)
    meshes.append(deg)                      # all-degenerate mesh, placed once
    meshes.append(dict(meshes[1]))          # unused mesh
    insts = list(s["instances"])
    ident = dict(insts[0])
    eye = np.eye(4, dtype=np.float32)
    ident.update(m=scenes.col_major(eye), inv=scenes.col_major(eye), n=np.eye(3, dtype=np.float32).reshape(9))
    insts.append(ident)
    placed = dict(insts[1])
    placed["mesh"] = len(meshes) - 2
    insts.append(placed)
    s = dict(s, meshes=meshes, instances=insts)
    osc = oracle.OracleScene(s)
    rng = np.random.default_rng(5)
    n = 40000
    o = rng.uniform(-10, 10, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    ctx.upload(s)
    ctx.build(width=2)
    flat = _trace(ctx, torch_cuda, o, d)
    ctx.build(width=1)
    info = ctx.info()
    assert info["nodes"] > 0
    _check_hits(ctx, torch_cuda, osc, o, d, 1e-4)
    two = _trace(ctx, torch_cuda, o, d)
    same = (two[0] == flat[0]) | ((two[0] >= 0) & (flat[0] >= 0) & (two[1] == flat[1]))
    assert same.all()
    film, _ = _render(ctx, s, 48, 40, 8, 6)
    ref, _ = osc.render(oracle.options(48, 40, 8, 6))
    assert rel_rmse(film, ref) <= REL_RMSE_TOL


def test_bake_bench_size_matches_oracle(ctx, oracle, torch_cuda):
    """The bake at the benchmark's size: the heightfield workload's 2048 x 1024 log-normal(0, 1.5)
    environment map to a 512 x 256 irradiance map, 128 samples per texel, against the oracle's CPU
    bake (rtol 1e-4)."""
    from axomae_b200 import scenes
    s = scenes.heightfield_scene(n=8, width=16, height=16, env_w=2048, env_h=1024, seed=0)
    env = next(t for t in s["textures"] if t["format"] == "f32")
    src = np.asarray(env["pixels"], np.float32).reshape(1024, 2048, 4)
    ts = torch_cuda.from_numpy(np.ascontiguousarray(src)).cuda()
    out = torch_cuda.zeros((256, 512, 4), dtype=torch_cuda.float32, device="cuda")
    ctx.bake_irradiance(ts.data_ptr(), 2048, 1024, 4, 512, 256, 128, out.data_ptr())
    ref = oracle.bake_irradiance(src, 512, 256, 128)
    np.testing.assert_allclose(out.cpu().numpy()[..., :3], ref[..., :3], rtol=1e-4, atol=1e-6)

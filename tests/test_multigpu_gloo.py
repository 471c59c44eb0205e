"""Sample-range partition and film reduction across ranks (axomae_b200.multigpu), run as gloo
process groups on the CPU.  Each rank's "render" is the oracle's per-sample radiance averaged over
the rank's sample range, the same quantity a GPU rank's film holds; the reduced film must equal the
mean over all samples computed in one process."""
import os
import socket

import numpy as np
import pytest

W, H, DEPTH = 12, 9, 3


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_film(osc, ob, spp_total, begin, count):
    opt = ob.options(W, H, spp_total, DEPTH)
    ys, xs = np.mgrid[0:H, 0:W]
    px, py = xs.reshape(-1), ys.reshape(-1)
    acc = np.zeros((px.size, 3), np.float64)
    for s in range(begin, begin + count):
        acc += osc.sample_radiance(opt, px, py, np.full(px.size, s))
    return (acc / max(count, 1)).astype(np.float32)


def _worker(rank, world, port, mode, per, out_dir):
    import torch
    import torch.distributed as dist
    import oracle_binding as ob
    from axomae_b200 import multigpu, scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = scenes.spheres_scene(W, H, n_spheres=6, seed=2)
        osc = ob.OracleScene(s)
        if mode == "weak":
            spp_total, begin, count = multigpu.weak_range(per, rank, world)
        else:
            spp_total, begin, count = multigpu.strong_range(per, rank, world)
        film = torch.from_numpy(_rank_film(osc, ob, spp_total, begin, count) if count else
                                np.zeros((W * H, 3), np.float32))
        multigpu.reduce_films(film, count)
        if rank == 0:
            np.save(os.path.join(out_dir, "reduced.npy"), film.numpy())
            full = _rank_film(osc, ob, spp_total, 0, spp_total)
            np.save(os.path.join(out_dir, "full.npy"), full)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("mode,world,per", [("weak", 2, 3), ("strong", 2, 7), ("strong", 3, 2)],
                         ids=["weak-2x3", "strong-7-over-2", "strong-2-over-3"])
def test_partitioned_render_equals_single_render(oracle, tmp_path, mode, world, per):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, mode, per, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    reduced = np.load(tmp_path / "reduced.npy")
    full = np.load(tmp_path / "full.npy")
    np.testing.assert_allclose(reduced, full, rtol=1e-5, atol=1e-6)


def _grad_worker(rank, world, port, per, out_dir):
    import torch
    import torch.distributed as dist
    import oracle_binding as ob
    from axomae_b200 import multigpu, scenes
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = scenes.spheres_scene(W, H, n_spheres=6, seed=2)
        n_tris = sum(np.size(s["meshes"][x["mesh"]]["indices"]) // 3 for x in s["instances"])
        n_mat = len(s["materials"])
        osc = ob.OracleScene(s)
        spp_total, begin, count = multigpu.strong_range(per, rank, world)
        opt = ob.options(W, H, spp_total, DEPTH, threads=2)
        d_image = np.random.default_rng(5).standard_normal((H, W, 4)).astype(np.float32)
        if count:
            ga, gr = osc.backward_range(opt, begin, count, d_image, n_tris, n_mat, threads=2)
        else:
            ga, gr = np.zeros((n_tris, 3), np.float32), np.zeros(n_mat, np.float32)
        ga_t, gr_t = torch.from_numpy(ga.copy()), torch.from_numpy(gr.copy())
        multigpu.reduce_gradients([ga_t, gr_t], count)
        if rank == 0:
            fa, fr = osc.backward(opt, d_image, n_tris, n_mat, threads=2)
            np.savez(os.path.join(out_dir, "grads.npz"), ga=ga_t.numpy(), gr=gr_t.numpy(), fa=fa, fr=fr)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,per", [(2, 4), (3, 2)], ids=["4-over-2", "2-over-3"])
def test_partitioned_gradients_equal_single_backward(oracle, tmp_path, world, per):
    """The replay adjoint split by sample range over gloo ranks, each rank's gradient reduced with
    reduce_gradients, equals the oracle's backward over all samples in one process (in "2-over-3"
    rank 0 has an empty range and contributes zeros)."""
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_grad_worker, args=(world, port, per, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    g = np.load(tmp_path / "grads.npz")
    assert np.abs(g["fa"]).max() > 0 and np.abs(g["fr"]).max() > 0
    np.testing.assert_allclose(g["ga"], g["fa"], rtol=1e-4, atol=1e-6 * np.abs(g["fa"]).max())
    np.testing.assert_allclose(g["gr"], g["fr"], rtol=1e-4, atol=1e-6 * np.abs(g["fr"]).max())


def test_ranges_cover_the_frame_once():
    from axomae_b200 import multigpu
    for world in (1, 2, 3, 8):
        for spp in (1, 5, 64):
            seen = []
            for r in range(world):
                tot, b, c = multigpu.strong_range(spp, r, world)
                assert tot == spp
                seen += list(range(b, b + c))
            assert seen == list(range(spp))
            tot, b, c = multigpu.weak_range(spp, world - 1, world)
            assert tot == spp * world and b + c == tot
    with pytest.raises(ValueError):
        multigpu.weak_range(0, 0, 1)
    with pytest.raises(ValueError):
        multigpu.strong_range(4, 2, 2)


def _failing_worker(rank, world, port, fail_rank, kind, out_dir):
    import datetime
    import torch
    import torch.distributed as dist
    from axomae_b200 import multigpu
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    try:
        failed = rank == fail_rank
        try:
            if kind == "films":
                multigpu.reduce_films(torch.full((16,), float("nan") if failed else 1.0), 1, failed=failed)
            else:
                multigpu.reduce_gradients([torch.ones(6), torch.ones(2)], 3, failed=failed)
            outcome = "returned"
        except multigpu.RankFailure as e:
            outcome = "raised: %s" % e
        # the ranks stay in step after the failure: one more reduction succeeds everywhere
        film = torch.full((4,), float(rank + 1))
        multigpu.reduce_films(film, 1)
        with open(os.path.join(out_dir, "rank%d.txt" % rank), "w") as f:
            f.write("%s\n%s\n" % (outcome, film.tolist()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["films", "gradients"])
def test_failed_rank_raises_on_every_rank(tmp_path, kind):
    """A rank whose render (or backward) failed reports it in the reduction: every rank raises
    RankFailure, none waits on a peer, and the next reduction works on all ranks."""
    import torch.multiprocessing as mp
    world = 3
    mp.start_processes(_failing_worker, args=(world, _free_port(), 1, kind, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        outcome, film = open(tmp_path / ("rank%d.txt" % r)).read().splitlines()
        assert outcome.startswith("raised: 1 rank(s)"), outcome
        assert film == str([2.0] * 4)  # mean of 1, 2, 3


def _vanishing_worker(rank, world, port, out_dir):
    import datetime
    import time
    import torch
    import torch.distributed as dist
    from axomae_b200 import multigpu
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        os._exit(0)  # the rank is lost between steps, with nothing in flight
    t0 = time.monotonic()
    try:
        multigpu.reduce_films(torch.ones(16), 1)
        outcome = "returned"
    except Exception as e:  # the process group reports the lost peer
        outcome = "raised %s" % type(e).__name__
    with open(os.path.join(out_dir, "rank0.txt"), "w") as f:
        f.write("%s\n%.1f\n" % (outcome, time.monotonic() - t0))
    os._exit(0)  # no destroy_process_group: its peer is gone


def test_lost_rank_ends_the_reduction_with_an_error(tmp_path):
    """A rank that leaves between steps: the survivor's next reduction ends with an error within the
    process group's short timeout instead of waiting for good."""
    import multiprocessing
    ctx = multiprocessing.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_vanishing_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    outcome, secs = open(tmp_path / "rank0.txt").read().splitlines()
    assert outcome.startswith("raised"), outcome
    assert float(secs) < 60

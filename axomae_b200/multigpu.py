"""Multi-GPU partition of a render by sample range (one process per GPU, torch.distributed).

Every rank renders the same frame over its own range of sample indices (the index mapping
(x * H + y) * spp_total + s keeps the samples disjoint and identical to a single-GPU render of
spp_total samples), then one all-reduce combines the films.  A rank's film is the mean of its
samples, so the combination weights each film by its sample count:

    mean = sum_r count_r * film_r / sum_r count_r

The differentiable render partitions the same way: a rank's backward gives the gradient of its own
film (the mean over its samples), so the gradient of the combined film is the count-weighted sum

    grad = sum_r count_r * grad_r / sum_r count_r

(one all-reduce of the 3 * triangles + materials parameter gradients).

The path has no other exchange: scenes and BVHs are built on every rank, and nothing crosses
between ranks while a frame renders.

Failures.  A rank whose render or backward failed still takes part in the reduction, with
`failed=True` (its film or gradients are replaced by zeros); the reduction carries the failure
count beside the sample count, and every rank then raises RankFailure, so all ranks take the same
collective steps and none waits for a peer that gave up.  A rank that dies or never arrives is
caught by the process group's timeout, which the caller keeps short (the collective then raises).
"""


class RankFailure(RuntimeError):
    """Raised on every rank after a reduction in which at least one rank reported a failure."""


def weak_range(spp_per_rank: int, rank: int, world: int):
    """Weak scaling: every rank adds spp_per_rank samples; returns (spp_total, sample_begin, count)."""
    if spp_per_rank <= 0 or not 0 <= rank < world:
        raise ValueError("bad sample partition")
    return spp_per_rank * world, rank * spp_per_rank, spp_per_rank


def strong_range(spp_total: int, rank: int, world: int):
    """Strong scaling: spp_total samples split as evenly as possible; returns (spp_total, begin, count).
    Ranks beyond spp_total get an empty range (count 0) and must skip the render but still take part
    in the reduction."""
    if spp_total <= 0 or not 0 <= rank < world:
        raise ValueError("bad sample partition")
    begin = rank * spp_total // world
    end = (rank + 1) * spp_total // world
    return spp_total, begin, end - begin


def _counts(count: int, failed: bool, device):
    import torch
    return torch.tensor([0.0 if failed else float(count), 1.0 if failed else 0.0], dtype=torch.float64,
                        device=device)


def _check(counts):
    ranks_failed = int(counts[1].item())
    if ranks_failed:
        raise RankFailure("%d rank(s) reported a failed render or backward" % ranks_failed)
    return counts[0].item()


def reduce_films(film, count: int, group=None, failed: bool = False):
    """In place: film (a float tensor, this rank's mean over `count` samples) becomes the mean over
    every rank's samples.  Collective: all ranks call it in the same order.  A rank whose render
    failed passes failed=True; then every rank raises RankFailure after the reduction."""
    import torch.distributed as dist
    counts = _counts(count, failed, film.device)
    if failed:
        film.zero_()
    else:
        film.mul_(float(count))
    dist.all_reduce(film, group=group)
    dist.all_reduce(counts, group=group)
    total = _check(counts)
    if total > 0:
        film.div_(total)
    return film


def reduce_gradients(grads, count: int, group=None, failed: bool = False):
    """In place: each tensor in `grads` (this rank's gradient of the mean over its `count` samples,
    e.g. per-triangle albedo and per-material roughness gradients) becomes the gradient of the mean
    over every rank's samples.  One all-reduce of the concatenated gradients, one of the counts.
    Collective: all ranks call it in the same order, with the same tensor shapes.  failed=True as
    in reduce_films."""
    import torch
    import torch.distributed as dist
    grads = list(grads)
    if not grads:
        return grads
    flat = torch.cat([g.reshape(-1) for g in grads]).to(torch.float32)
    counts = _counts(count, failed, flat.device)
    if failed:
        flat.zero_()
    else:
        flat.mul_(float(count))
    dist.all_reduce(flat, group=group)
    dist.all_reduce(counts, group=group)
    total = _check(counts)
    if total > 0:
        flat.div_(total)
    off = 0
    for g in grads:
        n = g.numel()
        g.copy_(flat[off:off + n].reshape(g.shape))
        off += n
    return grads

"""Sharding a batch of independent images over ranks, and the final gather.

Images are independent systems, so a batch is split across GPUs without any
exchange in the solve: each rank gets a subset whose pixel count is as even
as possible (longest-processing-time greedy on h*w), solves it with its own
batched launch, and only per-image results are gathered at the end: the
alphas and the per-image solve statistics go to rank 0, in batch order, in
one ``gather`` each (NCCL over NVLink for device tensors, gloo for host
tensors). There is no collective inside the solve.
"""

import torch

__all__ = ["shard_sizes", "gather_images", "solve_alpha_sharded", "STAT_FIELDS"]

# Per-image statistics carried by the gather, in this order.
STAT_FIELDS = ("iters", "status", "norm_r", "norm_b", "outer_iters")


def shard_sizes(sizes, world_size):
    """Assign images to ranks; returns one sorted index list per rank.

    ``sizes`` are ``(h, w)`` pairs. Deterministic: ties break by image index,
    so every rank computes the same assignment without communication.
    """
    if world_size <= 0:
        raise ValueError("world_size must be positive")
    order = sorted(range(len(sizes)), key=lambda k: (-(sizes[k][0] * sizes[k][1]), k))
    load = [0] * world_size
    parts = [[] for _ in range(world_size)]
    for k in order:
        r = min(range(world_size), key=lambda q: (load[q], q))
        parts[r].append(k)
        load[r] += sizes[k][0] * sizes[k][1]
    return [sorted(p) for p in parts]


def gather_images(local, sizes, parts, rank, world_size, device, dst=0, group=None):
    """Gather per-image arrays of every rank to rank ``dst``, in batch order.

    ``local``: this rank's arrays (tensors on ``device``), one per image of
    ``parts[rank]`` in that order; image ``k`` of the batch holds
    ``sizes[k]`` elements (an int or a shape). Every rank calls this with the
    same ``sizes`` and ``parts`` (``shard_sizes`` computes them without
    communication). Each rank sends one flat float64 buffer, padded to the
    largest rank's element count, through a single ``torch.distributed``
    ``gather``. Returns the list of all images (float64, flat, on ``device``)
    on ``dst`` and None elsewhere. With one rank nothing is communicated.
    """
    import torch.distributed as dist

    def numel(s):
        if isinstance(s, int):
            return s
        n = 1
        for d in s:
            n *= int(d)
        return n

    counts = [sum(numel(sizes[k]) for k in p) for p in parts]
    mine = parts[rank]
    if len(local) != len(mine):
        raise ValueError("rank %d holds %d images, its shard has %d" % (rank, len(local), len(mine)))
    for k, a in zip(mine, local):
        if a.numel() != numel(sizes[k]):
            raise ValueError("image %d: %d elements, expected %d" % (k, a.numel(), numel(sizes[k])))
    width = max(max(counts), 1)
    send = torch.zeros(width, dtype=torch.float64, device=device)
    off = 0
    for a in local:
        n = a.numel()
        send[off:off + n] = a.reshape(-1).to(torch.float64)
        off += n
    if world_size == 1:
        bufs = [send]
    else:
        bufs = ([torch.empty(width, dtype=torch.float64, device=device) for _ in range(world_size)]
                if rank == dst else None)
        dist.gather(send, gather_list=bufs, dst=dst, group=group)
        if rank != dst:
            return None
    out = [None] * len(sizes)
    for r, p in enumerate(parts):
        off = 0
        for k in p:
            n = numel(sizes[k])
            out[k] = bufs[r][off:off + n]
            off += n
    return out


def solve_alpha_sharded(images, trimaps, rank, world_size, device, dst=0, group=None, **kw):
    """Solve a batch of images split over ``world_size`` ranks (one per GPU).

    Every rank passes the whole batch (host arrays) and solves its own shard
    with ``solve_alpha`` on ``device``; the alphas (``(h, w)`` float64) and the
    per-image statistics (a ``(n_images, 5)`` float64 tensor, columns
    ``STAT_FIELDS``) are gathered to rank ``dst``. Returns ``(alphas, stats)``
    on ``dst`` and ``(None, None)`` elsewhere. ``kw`` goes to ``solve_alpha``.
    """
    from . import _device as devmod
    from .batch import solve_alpha

    sizes = [tuple(t.shape[:2]) for t in trimaps]
    parts = shard_sizes(sizes, world_size)
    mine = parts[rank]
    with torch.cuda.device(device):
        if mine:
            imgs = [devmod.to_device(images[k], torch.float64) for k in mine]
            tris = [devmod.to_device(trimaps[k], torch.float64) for k in mine]
            alphas, stats = solve_alpha(imgs, tris, return_stats=True, **kw)
        else:
            alphas, stats = [], []
        st = torch.tensor([[getattr(s, f) for f in STAT_FIELDS] for s in stats],
                          dtype=torch.float64).reshape(len(mine), len(STAT_FIELDS)).to(device)
        all_alphas = gather_images(alphas, sizes, parts, rank, world_size, device, dst, group)
        all_stats = gather_images(list(st), [len(STAT_FIELDS)] * len(sizes), parts, rank,
                                  world_size, device, dst, group)
    if all_alphas is None:
        return None, None
    alphas = [a.reshape(s) for a, s in zip(all_alphas, sizes)]
    return alphas, torch.stack(all_stats)

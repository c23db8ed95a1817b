"""Sharding a batch of independent images over ranks.

Images are independent systems, so a batch is split across GPUs without any
exchange in the solve: each rank gets a subset whose pixel count is as even
as possible (longest-processing-time greedy on h*w), solves it with its own
batched launch, and only per-image results are gathered at the end.
"""

__all__ = ["shard_sizes"]


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

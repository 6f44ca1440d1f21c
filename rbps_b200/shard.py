"""Splitting one set of independent worlds across ranks (one GPU each).

Batched worlds share no state, so a multi-GPU run needs no exchange on the
step path: each rank steps its own batch.  What must be decided is which
worlds go where.  A world's step cost grows with its body count, so the
split balances bodies, not world counts: largest world first, each to the
rank with the fewest bodies so far (ties to the lower rank), which leaves
every rank within one world's body count of every other.  Within a rank
the worlds keep their order in the set, so one rank holds the whole set in
its original order.
"""
import heapq

import numpy as np


def partition_worlds(body_counts, n_parts):
    """Indices of the worlds of each part: a list of n_parts sorted index
    arrays that together cover range(len(body_counts)) exactly once."""
    counts = np.asarray(body_counts, np.int64)
    if n_parts < 1:
        raise ValueError("partition_worlds: n_parts must be >= 1")
    heap = [(0, r) for r in range(n_parts)]
    parts = [[] for _ in range(n_parts)]
    # stable order: larger worlds first, index breaks ties
    for w in sorted(range(len(counts)), key=lambda i: (-int(counts[i]), i)):
        load, r = heapq.heappop(heap)
        parts[r].append(w)
        heapq.heappush(heap, (load + int(counts[w]), r))
    return [np.array(sorted(p), np.int64) for p in parts]


def shard_scene(scene, n_parts, part):
    """The scene restricted to the worlds of `part` (of n_parts)."""
    idx = partition_worlds([w.n_bodies for w in scene.worlds], n_parts)[part]
    return type(scene)(scene.name, scene.timestep, scene.substeps, scene.steps, [scene.worlds[i] for i in idx],
                       scene.description), idx

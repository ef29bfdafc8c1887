"""Statistics that judge a final layout by what it looks like.

ForceAtlas2 iterates chaotically: two runs whose forces differ by float
rounding drift apart node by node, so layouts are compared by the
distribution of their edge lengths and by their stress against graph
distances, not by coordinates.
"""
from __future__ import annotations

import numpy as np


def edge_lengths(xy, sources, targets) -> np.ndarray:
    """Euclidean length of every edge (float64)."""
    xy = np.asarray(xy, np.float64).reshape(-1, 2)
    d = xy[np.asarray(sources)] - xy[np.asarray(targets)]
    return np.sqrt((d ** 2).sum(1))


def stress(xy, sources, targets, n_src: int = 24, seed: int = 0) -> float:
    """Kamada-Kawai stress over all pairs (source, v) from n_src BFS sources,
    at the layout scale that minimises it: mean((a |p_u - p_v| - d)^2 / d^2),
    with a = sum(|p|/d) / sum(|p|^2/d^2) and d the hop distance."""
    from scipy.sparse import coo_matrix
    from scipy.sparse.csgraph import shortest_path
    xy = np.asarray(xy, np.float64).reshape(-1, 2)
    n = len(xy)
    a = coo_matrix((np.ones(len(sources)), (np.asarray(sources), np.asarray(targets))),
                   shape=(n, n)).tocsr()
    src = np.random.default_rng(seed).choice(n, min(n_src, n), replace=False)
    dist = shortest_path(a, directed=False, unweighted=True, indices=src)
    ok = np.isfinite(dist) & (dist > 0)
    rows, cols = np.nonzero(ok)
    d = dist[rows, cols]
    e = np.sqrt(((xy[src[rows]] - xy[cols]) ** 2).sum(1))
    scale = (e / d).sum() / ((e / d) ** 2).sum()
    return float((((scale * e - d) / d) ** 2).mean())


def summary(xy, sources, targets, n_src: int = 24) -> dict:
    """Mean edge length, its coefficient of variation, and stress."""
    lengths = edge_lengths(xy, sources, targets)
    return {"edge_len_mean": float(lengths.mean()),
            "edge_len_cv": float(lengths.std() / lengths.mean()),
            "stress": stress(xy, sources, targets, n_src)}

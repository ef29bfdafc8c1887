"""Seeded synthetic graphs with the shapes of the workloads the engine is measured on.

No public dataset is involved: every workload is generated here from a seed.

* ``rmat_edges``  -- R-MAT (Chakrabarti et al. 2004) edge draws, self-loops and
  repeated undirected edges removed, listed as sorted unique (lo, hi) pairs.
* ``ba_edges``    -- Barabasi-Albert preferential attachment (repeated-nodes
  method), m edges per new node.
* ``sbm_edges``   -- stochastic block model with equal blocks.

Each returns two uint32 arrays (sources, targets) in edge-list file order; the
engine's graph loader then assigns node ids by first appearance, as the
reference's ``RPGraph::UGraph`` does.
"""
from __future__ import annotations

import numpy as np


def _unique(x: np.ndarray) -> np.ndarray:
    """Sorted distinct values of an integer array (np.unique's result; a sort
    and a neighbour comparison, much faster than np.unique on large arrays)."""
    y = np.sort(x)
    if len(y) < 2:
        return y
    return y[np.concatenate(([True], y[1:] != y[:-1]))]


def _rmat_chunk_keys(args):
    """Keys (lo << scale | hi) of draws [start, start + m) of the R-MAT stream:
    the generator jumps ahead to the chunk's first random number (each level
    of a chunk takes m numbers, so draw block `start` begins at number
    start * scale)."""
    scale, start, m, a, b, c, seed = args
    bg = np.random.PCG64(seed)
    bg.advance(start * scale)
    rng = np.random.Generator(bg)
    src = np.zeros(m, np.int64)
    dst = np.zeros(m, np.int64)
    for lvl in range(scale):
        r = rng.random(m)
        sbit = r >= a + b
        dbit = ((r >= a) & (r < a + b)) | (r >= a + b + c)
        src |= sbit.astype(np.int64) << lvl
        dst |= dbit.astype(np.int64) << lvl
    keep = src != dst
    src, dst = src[keep], dst[keep]
    lo = np.minimum(src, dst)
    hi = np.maximum(src, dst)
    return _unique((lo << scale) | hi)


def rmat_edges(scale: int, n_draws: int, a: float = 0.57, b: float = 0.19,
               c: float = 0.19, seed: int = 0, chunk: int = 1 << 22,
               workers: int | None = None):
    """R-MAT draws over 2**scale ids: per level, quadrant (0,0) w.p. a, (0,1) b,
    (1,0) c, (1,1) d = 1-a-b-c.  Returns the unique undirected (lo, hi) pairs
    sorted ascending, self-loops dropped.  The draws come from one PCG64
    stream seeded with `seed`, in chunks of `chunk` draws level by level;
    chunks are generated by `workers` spawned processes (default: the CPU
    count when there are more than 8 chunks), each jumping the stream ahead to
    its chunk, so the result does not depend on the number of workers."""
    import os
    jobs = [(scale, start, min(chunk, n_draws - start), a, b, c, seed)
            for start in range(0, n_draws, chunk)]
    if workers is None:
        workers = min(32, os.cpu_count() or 1) if len(jobs) > 8 else 1
    if workers <= 1:
        keys = [_rmat_chunk_keys(j) for j in jobs]
    else:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(min(workers, len(jobs)),
                                 mp_context=mp.get_context("spawn")) as ex:
            keys = list(ex.map(_rmat_chunk_keys, jobs))
    k = _unique(np.concatenate(keys)) if len(keys) > 1 else keys[0]
    lo = (k >> scale).astype(np.uint32)
    hi = (k & ((1 << scale) - 1)).astype(np.uint32)
    return lo, hi


def ba_edges(n: int, m: int, seed: int = 0):
    """Barabasi-Albert: nodes m..n-1 each attach to m distinct earlier nodes
    chosen with probability proportional to degree (repeated-nodes list)."""
    rng = np.random.default_rng(seed)
    targets = list(range(m))
    repeated: list[int] = []
    src, dst = [], []
    for s in range(m, n):
        for t in targets:
            src.append(s)
            dst.append(t)
        repeated.extend(targets)
        repeated.extend([s] * m)
        chosen: set[int] = set()
        rep = np.asarray(repeated)
        while len(chosen) < m:
            for t in rep[rng.integers(0, len(rep), size=2 * m)]:
                if len(chosen) < m:
                    chosen.add(int(t))
        targets = sorted(chosen)
    return np.asarray(src, np.uint32), np.asarray(dst, np.uint32)


def sbm_edges(n: int, blocks: int, p_in: float, p_out: float, max_mean_degree: float,
              seed: int = 0):
    """Stochastic block model on n nodes in `blocks` equal blocks.  When the
    expected mean degree exceeds max_mean_degree both probabilities are scaled
    down to meet it.  Returns unique (lo, hi) pairs sorted ascending."""
    rng = np.random.default_rng(seed)
    size = n // blocks
    sizes = np.full(blocks, size, np.int64)
    sizes[: n - size * blocks] += 1
    bounds = np.concatenate([[0], np.cumsum(sizes)])
    exp_deg = p_in * (sizes.mean() - 1) + p_out * (n - sizes.mean())
    if exp_deg > max_mean_degree:
        s = max_mean_degree / exp_deg
        p_in, p_out = p_in * s, p_out * s
    los, his = [], []
    # within blocks
    for bi in range(blocks):
        b0, nb = bounds[bi], sizes[bi]
        pairs = nb * (nb - 1) // 2
        k = rng.binomial(pairs, p_in)
        if k:
            idx = _unique(rng.integers(0, pairs, size=k))
            # unrank pair index -> (i < j)
            i = (nb - 2 - np.floor(np.sqrt(-8.0 * idx + 4.0 * nb * (nb - 1) - 7) / 2.0 - 0.5)).astype(np.int64)
            j = idx + i + 1 - nb * (nb - 1) // 2 + (nb - i) * ((nb - i) - 1) // 2
            los.append(b0 + i)
            his.append(b0 + j)
    # between blocks: a binomial count per block pair, all pairs at once
    bi, bj = np.triu_indices(blocks, 1)
    if len(bi):
        pairs = sizes[bi] * sizes[bj]
        k = rng.binomial(pairs, p_out)
        which = np.repeat(np.arange(len(bi)), k)
        if len(which):
            idx = (rng.random(len(which)) * pairs[which]).astype(np.int64)
            idx = np.minimum(idx, pairs[which] - 1)
            key = _unique(which * (int(pairs.max()) + 1) + idx)
            which = key // (int(pairs.max()) + 1)
            idx = key % (int(pairs.max()) + 1)
            los.append(bounds[bi][which] + idx // sizes[bj][which])
            his.append(bounds[bj][which] + idx % sizes[bj][which])
    if not los:
        return np.zeros(0, np.uint32), np.zeros(0, np.uint32)
    lo = np.concatenate(los)
    hi = np.concatenate(his)
    k = _unique(lo * n + hi)
    return (k // n).astype(np.uint32), (k % n).astype(np.uint32)


def write_edgelist(path: str, src: np.ndarray, dst: np.ndarray) -> None:
    """Writes 'src dst' lines.  Numbers are right-aligned in fixed-width fields
    (leading spaces), which whitespace-skipping readers such as the
    reference's ``istringstream >> s >> t`` parse like plain numbers."""
    src = np.asarray(src, np.uint64)
    dst = np.asarray(dst, np.uint64)
    n = len(src)
    width = max(1, len(str(int(max(src.max(initial=0), dst.max(initial=0))))))
    line = 2 * width + 2
    buf = np.full((n, line), ord(" "), np.uint8)
    buf[:, -1] = ord("\n")
    for col0, vals in ((0, src), (width + 1, dst)):
        v = vals.copy()
        for d in range(width - 1, -1, -1):
            digit = (v % 10).astype(np.uint8) + ord("0")
            nz = (v > 0) | (d == width - 1)
            buf[:, col0 + d] = np.where(nz, digit, ord(" "))
            v //= 10
    with open(path, "wb") as f:
        f.write(buf.tobytes())


def _sbm_batch_part(args):
    out = []
    for n, b, s in args:
        lo, hi = sbm_edges(int(n), int(b), 0.05, 0.002, 40.0, seed=int(s))
        out.append((int(n), lo, hi))
    return out


def sbm_batch(num_graphs: int = 4096, n_min: int = 50, n_max: int = 20000, seed: int = 0,
              workers: int | None = None):
    """The batched workload: num_graphs stochastic block models with node
    counts log-uniform in [n_min, n_max], 2-32 equal blocks, p_in 0.05,
    p_out 0.002, mean degree capped at 40.  Returns (n, lo, hi) per graph.
    Graph i depends only on (seed, i); `workers` processes (spawned, default
    the CPU count) generate them."""
    import os
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(n_min), np.log(n_max), num_graphs)).round().astype(np.int64)
    blocks = rng.integers(2, 33, num_graphs)
    jobs = [(int(sizes[i]), int(min(blocks[i], sizes[i])), seed * 100003 + i)
            for i in range(num_graphs)]
    workers = workers or min(32, os.cpu_count() or 1)
    if workers <= 1 or num_graphs < 64:
        return _sbm_batch_part(jobs)
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    chunks = [jobs[w::workers] for w in range(workers)]
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        parts = list(ex.map(_sbm_batch_part, chunks))
    out = [None] * num_graphs
    for w, part in enumerate(parts):
        for j, g in enumerate(part):
            out[w + j * workers] = g
    return out

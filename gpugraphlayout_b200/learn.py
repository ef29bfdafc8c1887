"""Training the learned far-field correction on layouts the engine produces.

The recipe: lay a training graph out with the plain walk from random
positions; after `warmup` iterations take `snapshots` layouts, `every`
iterations apart; at each, walk the tree at the theta (and multipole order)
the correction is meant for and collect every (group, cell) pair's features
and exact FP64 target (fa2_learn_collect); then fit the MLP with the
training kernels (fa2_learn_fit).  Everything runs on the GPU through the
C ABI; the samples stay in device memory.
"""
from __future__ import annotations

import time

from . import Engine, FarFieldMLP, LearnSet, random_positions


def train_correction(num_nodes: int, sources, targets, *, theta: float, multipole: int = 1,
                     strong_gravity: bool = True, gravity: float = 1.0, scale: float = 10.0,
                     width: float = 2.0e4, seed: int = 1234, warmup: int = 20,
                     snapshots: int = 200, every: int = 2, capacity: int = 60_000_000,
                     steps: int = 4000, batch: int = 4096, lr: float = 2e-3,
                     init_seed: int = 0, device: int = 0):
    """Returns (mlp, info): the trained FarFieldMLP and a dict with the
    sample count, the last batch loss and the seconds spent collecting and
    fitting."""
    e = Engine(num_nodes, sources, targets, strong_gravity=strong_gravity, gravity=gravity,
               scale=scale, device=device)
    e.set_positions(random_positions(num_nodes, width, width, seed))
    e.step(warmup)
    ls = LearnSet(capacity, device=device)
    t0 = time.perf_counter()
    for _ in range(snapshots):
        e.step(every)
        ls.collect(e, theta, multipole)
    t1 = time.perf_counter()
    mlp = FarFieldMLP(seed=init_seed)
    loss = ls.fit(mlp, steps=steps, batch=batch, lr=lr, seed=init_seed + 1)
    t2 = time.perf_counter()
    info = {"samples": len(ls), "snapshots": snapshots, "every": every, "warmup": warmup,
            "theta": theta, "multipole": multipole, "fit_steps": steps, "batch": batch,
            "final_loss": loss, "collect_s": t1 - t0, "fit_s": t2 - t1}
    ls.close()
    e.close()
    return mlp, info

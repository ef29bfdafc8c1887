"""Generates the golden fixtures in this directory from the reference's own code.

Each fixture is the output of the reference run here, not of this project's
engine or oracle:
  * ``step_*.npz``: the reference's CUDA kernels (src/RPBHKernels.cu,
    src/RPFA2Kernels.cu) executed by the CPU SIMT emulator in oracle/_ref, in
    CUDAForceAtlas2::doStep order, on a seeded graph and positions: body sort
    order (sortd), gravity+attraction and total forces before displacement,
    positions and adaptive speed after each of three steps;
  * ``ugraph_*.npz``: the reference's RPGraph::UGraph loader on an edge-list
    text with comments, self-loops, repeated and reversed edges.

Run from the repository root after `make -C oracle ref` (needs the reference
sources):  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from gpugraphlayout_b200 import synth  # noqa: E402
from oracle import oracle as O  # noqa: E402

UGRAPH_TEXT = (
    "# edge list with the cases the loader must handle\n"
    "5 3\n3 5\n7 7\n9 5\n# comment\n5 3\n1\t9\n12 3\r\n3 12\n100 1\n1 100\n"
    "  4   8  \n8 4 trailing words\n6 2\n2 6\n42 7\n"
)


def step_fixture(name, g, xy, k_r, k_g, sg, steps=3):
    em = O.RefGPUEmu(g, xy, k_r, k_g, sg, tree_threads=32)
    out = {"sources": g.sources, "targets": g.targets, "mass": g.mass,
           "xy0": np.asarray(xy, np.float32), "k_r": np.float32(k_r), "k_g": np.float32(k_g),
           "strong_gravity": np.int32(sg)}
    for it in range(steps):
        em.step()
        out[f"sortd_{it}"] = em.sortd.copy()
        out[f"f_ga_{it}"] = em.f_ga.reshape(-1, 2).copy()
        out[f"f_tot_{it}"] = em.f_tot.reshape(-1, 2).copy()
        out[f"xy_{it}"] = em.positions().copy()
        out[f"speed_{it}"] = np.float32(em.global_speed)
        out[f"speed_eff_{it}"] = np.float32(em.speed_efficiency)
    del em
    np.savez_compressed(os.path.join(HERE, f"step_{name}.npz"), **out)


def main():
    s, t = synth.ba_edges(1500, 3, seed=11)
    g = O.Graph(s, t)
    step_fixture("ba1500_sg", g, O.random_positions(g.n, 2000, 2000, 1234), 10.0, 1.0, True)
    step_fixture("ba1500_wg", g, O.random_positions(g.n, 2000, 2000, 77), 80.0, 1.0, False)
    s, t = synth.sbm_edges(1200, 4, 0.05, 0.002, 40, seed=5)
    g = O.Graph(s, t)
    rng = np.random.default_rng(9)
    centres = rng.uniform(-800, 800, size=(4, 2))
    xy = (centres[np.arange(g.n) % 4] + rng.normal(0, 4.0, size=(g.n, 2))).astype(np.float32)
    step_fixture("sbm1200_clustered", g, xy, 2.0, 1.0, False)

    path = os.path.join(HERE, "ugraph_cases.txt")
    with open(path, "w") as f:
        f.write(UGRAPH_TEXT)
    rg = O.RefGraph(path)
    off, adj = rg.adjacency()
    np.savez_compressed(os.path.join(HERE, "ugraph_cases.npz"), node_map_r=rg.node_map_r(),
                        degrees=rg.degrees(), adj_offsets=off, adj=adj)


if __name__ == "__main__":
    main()

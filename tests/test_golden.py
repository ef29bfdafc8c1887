"""Committed golden fixtures (tests/golden, made by make_golden.py from the
reference's own kernels and loader) against the oracle (bit for bit, CPU) and
against the CUDA engine (sort order bit for bit, forces and positions within
the tolerances of test_gpu_parity, GPU)."""
import glob
import os

import numpy as np
import pytest

from conftest import ROOT, rel_rmse

GOLDEN = os.path.join(ROOT, "tests", "golden")
STEP_FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "step_*.npz")))


def _graph(z):
    class G:
        pass
    g = G()
    g.sources = z["sources"]
    g.targets = z["targets"]
    g.mass = z["mass"]
    g.n = len(g.mass)
    g.m = len(g.sources)
    return g


@pytest.mark.parametrize("path", STEP_FIXTURES, ids=os.path.basename)
def test_oracle_reproduces_golden_steps(path):
    from oracle import oracle as O
    z = np.load(path)
    g = _graph(z)
    fo = O.FA2(g, z["xy0"], float(z["k_r"]), float(z["k_g"]), bool(z["strong_gravity"]))
    for it in range(3):
        fo.step()
        assert np.array_equal(fo.sortd, z[f"sortd_{it}"])
        assert np.array_equal(fo.f_ga.reshape(-1, 2), z[f"f_ga_{it}"])
        assert np.array_equal(fo.f_tot.reshape(-1, 2), z[f"f_tot_{it}"])
        assert np.array_equal(fo.positions, z[f"xy_{it}"])
        assert np.float32(fo.global_speed) == z[f"speed_{it}"]


def test_ugraph_reproduces_golden_loader():
    from gpugraphlayout_b200 import UGraph
    z = np.load(os.path.join(GOLDEN, "ugraph_cases.npz"))
    g = UGraph(os.path.join(GOLDEN, "ugraph_cases.txt"))
    assert np.array_equal(g.node_map_r, z["node_map_r"])
    assert np.array_equal(g.degrees(), z["degrees"])
    s, t = g.edges()
    assert np.array_equal(t, z["adj"])
    assert np.array_equal(s, np.repeat(np.arange(len(z["degrees"])), np.diff(z["adj_offsets"])))


@pytest.mark.gpu
@pytest.mark.parametrize("path", STEP_FIXTURES, ids=os.path.basename)
def test_engine_reproduces_golden_steps(path):
    """Step 0 starts from the fixture's positions: sort order bit for bit.
    Later steps start from positions that already differ from the reference's
    by float rounding (summation order), so the sort order is checked as what
    it is, a function of the positions: the reference tree of the engine's own
    positions before the step.  Forces and positions stay within tolerance."""
    from gpugraphlayout_b200 import Engine
    from oracle import oracle as O
    z = np.load(path)
    g = _graph(z)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=bool(z["strong_gravity"]),
               gravity=float(z["k_g"]), scale=float(z["k_r"]))
    e.set_positions(z["xy0"])
    for it in range(3):
        before = e.get_positions()
        e.step(1)
        if it == 0:
            assert np.array_equal(e.sort_order(), z["sortd_0"].astype(np.uint32))
        else:
            expect = O.Tree(before, g.mass).sort().astype(np.uint32)
            assert np.array_equal(e.sort_order(), expect), it
        tot, ga = e.forces()
        tol = 1e-4 if it == 0 else 1e-3
        assert rel_rmse(ga, z[f"f_ga_{it}"]) <= tol / 10
        assert rel_rmse(tot, z[f"f_tot_{it}"]) <= tol
        assert e.stats()["global_speed"] == pytest.approx(float(z[f"speed_{it}"]), rel=1e-3)
    assert rel_rmse(e.get_positions(), z["xy_2"]) <= 1e-4

"""prevent_overlap in the oracle (CPU), against a float64 restatement of the
ForceAtlas2 paper's rule (Jacomy et al., PLoS ONE 2014).  The reference
declares the option (src/RPForceAtlas2.hpp:44) and exits on it
(src/RPCPUForceAtlas2.cpp:201-205), so the paper is the specification.

With theta small enough that the walk opens every cell, every interaction
is body to body, so the walk's repulsion is the direct sum of the rule."""
import numpy as np


def _graph(n=400, seed=2):
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(n, 3, seed=seed)
    return O.Graph(s, t)


def _sizes(n, seed=3):
    return np.random.default_rng(seed).uniform(0.0, 30.0, n).astype(np.float32)


def test_overlap_attraction_matches_float64_rule():
    from oracle import oracle as O
    g = _graph()
    xy = O.random_positions(g.n, 600, 600, 5)
    sz = _sizes(g.n)
    got = O.gravity_attraction(g, xy, 0.0, True, sizes=sz)
    p = xy.astype(np.float64)
    want = np.zeros((g.n, 2))
    for s, t in zip(g.sources, g.targets):
        v = p[t] - p[s]
        d = np.sqrt((v ** 2).sum())
        dp = d - sz[s] - sz[t]
        f = v * (dp / d) if dp > 0 else 0.0 * v
        want[s] += f
        want[t] -= f
    err = np.sqrt(((got - want) ** 2).sum() / (want ** 2).sum())
    assert err < 1e-5
    # some edges overlap at these sizes, some do not
    d = np.sqrt(((p[g.targets] - p[g.sources]) ** 2).sum(1))
    gap = d - sz[g.sources] - sz[g.targets]
    assert (gap < 0).any() and (gap > 0).any()


def test_overlap_repulsion_matches_direct_float64_sum():
    from oracle import oracle as O
    g = _graph()
    xy = O.random_positions(g.n, 600, 600, 5)
    sz = _sizes(g.n)
    tree = O.Tree(xy, g.mass)
    k_r, eps = 10.0, float(np.float32(0.05 * 0.05))
    got, ovf, _ = tree.repulsion(k_r, itolsq=1e12, sizes=sz)
    assert not ovf
    p = tree.xy.reshape(-1, 2).astype(np.float64)
    m = g.mass.astype(np.float64)
    d = p[:, None, :] - p[None, :, :]
    ds = np.sqrt((d ** 2).sum(2) + eps)
    dp = ds - sz[:, None] - sz[None, :]
    c = np.where(dp > 0, m[None, :] / (ds * np.where(dp > 0, dp, 1.0)),
                 np.where(dp < 0, 100.0 * m[None, :] / ds, 0.0))
    np.fill_diagonal(c, 0.0)
    want = k_r * m[:, None] * (c[:, :, None] * d).sum(1)
    err = np.sqrt(((got - want) ** 2).sum() / (want ** 2).sum())
    assert err < 1e-4


def test_zero_sizes_give_the_plain_rule():
    from oracle import oracle as O
    g = _graph()
    xy = O.random_positions(g.n, 600, 600, 5)
    tree = O.Tree(xy, g.mass)
    plain, _, _ = tree.repulsion(10.0)
    zero, _, _ = tree.repulsion(10.0, sizes=np.zeros(g.n, np.float32))
    err = np.sqrt(((plain - zero) ** 2).sum() / (plain ** 2).sum())
    assert err < 1e-5
    ga = O.gravity_attraction(g, xy, 1.0, True)
    ga0 = O.gravity_attraction(g, xy, 1.0, True, sizes=np.zeros(g.n, np.float32))
    assert np.sqrt(((ga - ga0) ** 2).sum() / (ga ** 2).sum()) < 1e-5

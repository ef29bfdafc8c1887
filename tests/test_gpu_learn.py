"""The learned far-field correction (fa2_mlp_*, fa2_learn_*,
fa2_set_learned_correction) through the C ABI.

* The tensor-core inference kernel against a PyTorch FP32 MLP with the same
  BF16-rounded weights and BF16-rounded hidden activations: relative RMSE
  at most 1e-2 (the accumulation order differs; in practice far below).
* One and two steps of the training kernels against PyTorch autograd and
  torch.optim.Adam on the same weighted loss: loss and first moment within
  1e-5 relative, the parameter update and the second moment (squared
  gradients) within 1e-4, the noise of another summation order.
* An all-zero MLP leaves the iteration exactly as the plain walk computes it:
  positions after several steps bit for bit, for both walks.
* Trained on the engine's own layouts (FP64 targets), the correction lowers
  the walk's error against the exact FP64 pairwise sum at a larger theta.
"""
import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu


def _torch_mlp(mlp, bf16):
    import torch
    layers = []
    for w, b in (("w1", "b1"), ("w2", "b2"), ("w3", "b3")):
        W = torch.tensor(mlp[w])
        if bf16:
            W = W.bfloat16().float()
        layers.append((W, torch.tensor(mlp[b])))
    return layers


def _torch_forward(layers, x, bf16):
    import torch
    h = torch.tensor(x)
    if bf16:
        h = h.bfloat16().float()
    for i, (W, b) in enumerate(layers):
        h = h @ W.T + b
        if i < 2:
            h = torch.relu(h)
            if bf16:
                h = h.bfloat16().float()
    return h.numpy()


@pytest.mark.parametrize("n", [1, 127, 128, 1000, 70000])
def test_inference_kernel_matches_torch_bf16_mlp(n):
    from gpugraphlayout_b200 import FarFieldMLP
    rng = np.random.default_rng(n)
    mlp = FarFieldMLP(seed=5)
    # larger weights than the initial ones, so the hidden layers do work
    for name in ("w1", "w2", "w3"):
        mlp[name] = mlp[name] * 3.0
    x = rng.normal(0.0, 1.0, (n, 12)).astype(np.float32)
    got = mlp.forward(x)
    want = _torch_forward(_torch_mlp(mlp, bf16=True), x, bf16=True)
    assert got.shape == (n, 2)
    assert np.isfinite(got).all()
    assert rel_rmse(got, want) <= 1e-2
    # the BF16 rounding of the hidden activations is the only difference
    # left: far below the bar
    assert rel_rmse(got, want) <= 2e-3


def test_inference_rows_are_independent():
    """Each row's output depends on that row alone (tiles of 128 rows, many
    blocks): a row gives the same bits at any position in the batch."""
    from gpugraphlayout_b200 import FarFieldMLP
    rng = np.random.default_rng(1)
    mlp = FarFieldMLP(seed=2)
    x = rng.normal(0.0, 1.0, (5000, 12)).astype(np.float32)
    a = mlp.forward(x)
    b = mlp.forward(x[::-1].copy())[::-1]
    assert np.array_equal(a, b)
    assert np.array_equal(mlp.forward(x[4321:4322]), a[4321:4322])


def _torch_train(mlp, x, t, w, lr, steps):
    import torch
    net = torch.nn.Sequential(torch.nn.Linear(12, 64), torch.nn.ReLU(), torch.nn.Linear(64, 64),
                              torch.nn.ReLU(), torch.nn.Linear(64, 2))
    with torch.no_grad():
        for li, (wn, bn) in zip((0, 2, 4), (("w1", "b1"), ("w2", "b2"), ("w3", "b3"))):
            net[li].weight.copy_(torch.tensor(mlp[wn]))
            net[li].bias.copy_(torch.tensor(mlp[bn]))
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    X, T = torch.tensor(x), torch.tensor(t)
    W = torch.tensor(np.minimum(w, 100.0).astype(np.float32))
    losses = []
    for _ in range(steps):
        loss = (W[:, None] * (net(X) - T) ** 2).mean()
        losses.append(float(loss.detach()))
        opt.zero_grad()
        loss.backward()
        opt.step()
    params = np.concatenate([p.detach().numpy().ravel() for p in net.parameters()])
    state = [opt.state[p] for p in net.parameters()]
    m = np.concatenate([s["exp_avg"].numpy().ravel() for s in state])
    v = np.concatenate([s["exp_avg_sq"].numpy().ravel() for s in state])
    return params, m, v, losses


@pytest.mark.parametrize("n", [300, 4096])
def test_training_steps_match_torch_adam(n):
    from gpugraphlayout_b200 import FarFieldMLP
    rng = np.random.default_rng(7 + n)
    mlp = FarFieldMLP(seed=9)
    x = rng.normal(0.0, 1.0, (n, 12)).astype(np.float32)
    t = rng.normal(0.0, 0.3, (n, 2)).astype(np.float32)
    w = rng.uniform(0.0, 3.0, n).astype(np.float32)
    w[::17] = 250.0  # past the weight cap
    p0 = mlp.vector()
    want_p, want_m, want_v, want_loss = _torch_train(mlp, x, t, w, 1e-3, 2)
    m, v = FarFieldMLP(seed=None), FarFieldMLP(seed=None)
    loss1 = mlp.train_step(m, v, 1, 1e-3, x, t, w)
    loss2 = mlp.train_step(m, v, 2, 1e-3, x, t, w)
    assert loss1 == pytest.approx(want_loss[0], rel=1e-5)
    assert loss2 == pytest.approx(want_loss[1], rel=1e-5)
    got_p = mlp.vector()
    # the update itself, not just the (much larger) parameters, must agree
    assert rel_rmse(got_p - p0, want_p - p0) <= 1e-4
    assert rel_rmse(m.vector(), want_m) <= 1e-5
    # v holds squared gradients: twice the gradients' summation-order noise
    assert rel_rmse(v.vector(), want_v) <= 1e-4


def _graph(n=6000, seed=3):
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(n, 3, seed=seed)
    return O.Graph(s, t)


@pytest.mark.parametrize("multipole", [1, 2])
def test_zero_correction_is_the_plain_walk_bit_for_bit(multipole):
    from gpugraphlayout_b200 import Engine, FarFieldMLP
    from oracle import oracle as O
    g = _graph()
    xy = O.random_positions(g.n, 2000, 2000, 11)
    runs = []
    for learned in (False, True):
        e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0, theta=1.5,
                   multipole=multipole)
        e.set_positions(xy)
        if learned:
            e.set_learned_correction(FarFieldMLP(seed=None))
        e.step(6)
        tot, ga = e.forces()
        runs.append((e.get_positions(), tot, e.stats()["global_speed"]))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])
    assert runs[0][2] == runs[1][2]


def test_trained_correction_lowers_the_error_against_fp64():
    """Samples from the engine's own layouts of one graph (every 4th step of
    a plain run), trained with the training kernels, then the corrected walk
    at theta 1.5 on a later layout: its repulsion error against the exact
    FP64 sum is below the plain walk's at the same theta."""
    from gpugraphlayout_b200 import Engine, FarFieldMLP, LearnSet
    from oracle import oracle as O
    g = _graph(20000, seed=5)
    xy = O.random_positions(g.n, 20000, 20000, 1234)
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0)
    e.set_positions(xy)
    e.step(20)
    ls = LearnSet(4_000_000)
    for _ in range(24):
        e.step(4)
        assert ls.collect(e, 1.5, 1) > 0
    f, t, w = ls.read(0, min(len(ls), 10000))
    assert np.isfinite(f).all() and np.isfinite(t).all() and (w > 0).all()
    mlp = FarFieldMLP(seed=0)
    loss = ls.fit(mlp, steps=1500, batch=4096, lr=2e-3, seed=1)
    assert np.isfinite(loss)
    e.step(30)
    P = e.get_positions()
    samples = np.arange(0, g.n, 7, dtype=np.uint32)
    exact = e.exact_repulsion(samples)
    errs = {}
    for name, learned in (("plain", None), ("learned", mlp)):
        e.set_approximation(1.5, 1)
        e.set_learned_correction(learned)
        e.set_positions(P)
        e.step(1)
        tot, ga = e.forces()
        errs[name] = rel_rmse((tot - ga)[samples], exact)
    e.set_learned_correction(None)
    assert errs["learned"] < 0.8 * errs["plain"], errs


def test_any_mlp_keeps_the_layout_finite():
    """An untrained MLP with large weights on a graph whose trees reach deep
    levels: each pair's correction is held to its cell's point-mass term and
    non-finite outputs add nothing, so 30 steps leave finite positions and
    no device error."""
    from gpugraphlayout_b200 import Engine, FarFieldMLP, synth
    from oracle import oracle as O
    s, t = synth.rmat_edges(16, 1 << 20, seed=0)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 2e4, 2e4, 1234)
    mlp = FarFieldMLP(seed=4)
    for name in ("w1", "w2", "w3", "b3"):
        mlp[name] = mlp[name] * 40.0
    e = Engine(g.n, g.sources, g.targets, strong_gravity=True, scale=10.0, theta=1.2)
    e.set_positions(xy)
    e.set_learned_correction(mlp)
    e.step(30)
    assert np.isfinite(e.get_positions()).all()
    st = e.stats()
    assert st["device_error"] == 0 and st["learned_pairs"] > 0

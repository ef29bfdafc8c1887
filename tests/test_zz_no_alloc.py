"""fa2_repulsion_noalloc (all scratch in a static device array, nothing
allocated per call) against the repulsion of fa2_step on the same positions
and masses, through the C ABI.

fa2_step's forces come back as the total and the gravity + attraction part;
their difference is the repulsion, rounded once more by the subtraction, so
the comparison is a relative RMSE of at most 1e-5 (the same tree, cell tests
and walk order give the same terms).  Two calls in a row, on different
positions, check that each call starts from cleared scratch.  Its name sorts
last, so pytest collects it after every other test file; it also passes on
its own in a fresh process, where its first call does the per-device set-up.

The entry point exists for callers that may not allocate device memory at the
call: code with a fixed device-memory budget, or a library running inside a
host framework whose caching allocator it must not disturb.  After the first
call on a device, neither torch's allocator nor the device's free memory
(cudaMemGetInfo) may change across calls.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_rmse

pytestmark = pytest.mark.gpu

TOL = 1e-5


def _params(scale):
    from gpugraphlayout_b200 import _native
    prm = _native.Params()
    _native.lib().fa2_default_params(C.byref(prm))
    prm.scale = scale
    return prm


def _noalloc(xy_dev, mass_dev, out_dev, prm, n=None):
    from gpugraphlayout_b200 import _native
    n = xy_dev.shape[0] if n is None else n
    return _native.lib().fa2_repulsion_noalloc(
        C.c_void_p(xy_dev.data_ptr()), C.c_void_p(mass_dev.data_ptr()), n, C.byref(prm), None,
        C.c_void_p(out_dev.data_ptr()))


def _step_repulsion(g, xy, scale):
    from gpugraphlayout_b200 import Engine
    e = Engine(g.n, g.sources, g.targets, strong_gravity=False, gravity=1.0, scale=scale)
    e.set_positions(xy)
    e.step(1)
    tot, ga = e.forces()
    return tot - ga


def test_noalloc_matches_step_on_two_calls_in_a_row():
    """The largest accepted size, then a smaller graph: the second call must
    not see anything the first one left in the scratch."""
    import torch
    from gpugraphlayout_b200 import _native, synth
    from oracle import oracle as O
    prm = _params(10.0)
    for n, seed in ((_native.FA2_NOALLOC_MAX_BODIES, 11), (3000, 12)):
        s, t = synth.ba_edges(n, 3, seed=seed)
        g = O.Graph(s, t)
        assert g.n == n
        xy = O.random_positions(g.n, 2000, 2000, seed)
        out = torch.full((g.n, 2), float("nan"), dtype=torch.float32, device="cuda")
        mass = torch.from_numpy(g.mass).cuda()
        assert _noalloc(torch.from_numpy(xy).cuda(), mass, out, prm) == 0
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        assert rel_rmse(got, _step_repulsion(g, xy, 10.0)) <= TOL, n


def test_noalloc_rejects_more_bodies_than_its_scratch_holds():
    import torch
    from gpugraphlayout_b200 import _native
    n = _native.FA2_NOALLOC_MAX_BODIES + 1
    xy = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    mass = torch.ones(n, dtype=torch.float32, device="cuda")
    out = torch.full((n, 2), 7.0, dtype=torch.float32, device="cuda")
    assert _noalloc(xy, mass, out, _params(1.0)) == 6  # FA2_ERR_TOO_LARGE
    assert bool((out == 7.0).all())  # nothing ran


def test_noalloc_reports_inputs_it_does_not_handle():
    """Coincident bodies (fa2_step would move them apart) and masses that are
    not whole numbers below 2^24 (fa2_step's are degree + 1) are refused with
    FA2_ERR_INVALID_ARGUMENT; the next call works again."""
    import torch
    from oracle import oracle as O
    n = 500
    xy = O.random_positions(n, 100, 100, 3)
    mass = torch.ones(n, dtype=torch.float32, device="cuda")
    out = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    prm = _params(1.0)
    same = xy.copy()
    same[7] = same[3]
    assert _noalloc(torch.from_numpy(same).cuda(), mass, out, prm) == 1
    frac = mass.clone()
    frac[11] = 1.5
    assert _noalloc(torch.from_numpy(xy).cuda(), frac, out, prm) == 1
    assert _noalloc(torch.from_numpy(xy).cuda(), mass, out, prm) == 0
    assert bool(torch.isfinite(out).all())


def test_noalloc_refuses_non_finite_positions():
    """A NaN or infinite position is flagged by the bounding-box pass and
    refused with FA2_ERR_INVALID_ARGUMENT before a tree is built."""
    import torch
    from oracle import oracle as O
    n = 700
    mass = torch.ones(n, dtype=torch.float32, device="cuda")
    out = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    prm = _params(1.0)
    for bad in (np.nan, np.inf):
        xy = O.random_positions(n, 100, 100, 3)
        xy[100, 1] = bad
        assert _noalloc(torch.from_numpy(xy).cuda(), mass, out, prm) == 1
    xy = O.random_positions(n, 100, 100, 3)
    assert _noalloc(torch.from_numpy(xy).cuda(), mass, out, prm) == 0
    assert bool(torch.isfinite(out).all())


def test_noalloc_leaves_device_memory_untouched_after_the_first_call():
    """Calls after the first neither allocate through torch's caching
    allocator nor change the device's free memory (cudaMemGetInfo)."""
    import torch
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(4000, 3, seed=21)
    g = O.Graph(s, t)
    xy = torch.from_numpy(O.random_positions(g.n, 2000, 2000, 21)).cuda()
    mass = torch.from_numpy(g.mass).cuda()
    out = torch.empty((g.n, 2), dtype=torch.float32, device="cuda")
    prm = _params(10.0)
    assert _noalloc(xy, mass, out, prm) == 0  # set-up and first kernel loads
    torch.cuda.synchronize()
    first = out.clone()
    alloc0 = torch.cuda.memory_allocated()
    reserved0 = torch.cuda.memory_reserved()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert _noalloc(xy, mass, out, prm) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert torch.cuda.memory_allocated() == alloc0
    assert torch.cuda.memory_reserved() == reserved0
    assert free1 == free0
    assert torch.equal(out, first)  # and every call gives the same bits


def test_noalloc_refuses_other_multipole_orders():
    """multipole 2 (the quadrupole walk) is not offered here; 0 or less is
    not a multipole order at all."""
    import torch
    n = 100
    xy = torch.zeros((n, 2), dtype=torch.float32, device="cuda")
    mass = torch.ones(n, dtype=torch.float32, device="cuda")
    out = torch.full((n, 2), 7.0, dtype=torch.float32, device="cuda")
    for mp, status in ((2, 7), (0, 1), (-1, 1)):  # FA2_ERR_UNSUPPORTED, _INVALID_ARGUMENT
        prm = _params(1.0)
        prm.multipole = mp
        assert _noalloc(xy, mass, out, prm) == status, mp
    assert bool((out == 7.0).all())  # nothing ran

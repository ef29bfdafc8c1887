"""Edge weight influence on the host, no GPU needed: the ctypes declarations
match include/fa2b200.h, fa2_create checks weights and delta before it looks
for a device, and the oracle's weighted attraction restates w^delta times the
unweighted force."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

LAYOUT_PROBE = r"""
#include <stddef.h>
#include <stdio.h>
#include "fa2b200.h"
int main(void) {
    printf("%zu %zu %zu %zu\n", sizeof(fa2_graph_desc), offsetof(fa2_graph_desc, weights),
           sizeof(fa2_params), offsetof(fa2_params, delta));
    return 0;
}
"""


def test_struct_layout_matches_header(tmp_path):
    from gpugraphlayout_b200 import _native as N
    src = tmp_path / "probe.c"
    src.write_text(LAYOUT_PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(exe), str(src)],
                   check=True)
    got = [int(v) for v in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got == [C.sizeof(N.GraphDesc), N.GraphDesc.weights.offset, C.sizeof(N.Params),
                   N.Params.delta.offset]


def _create_status(weights, delta):
    from gpugraphlayout_b200 import _native as N
    L = N.lib()
    s = np.array([0, 1, 2], np.uint32)
    t = np.array([1, 2, 0], np.uint32)
    w = None if weights is None else np.ascontiguousarray(weights, np.float32)
    g = N.GraphDesc(3, 3, s.ctypes.data, t.ctypes.data, None if w is None else w.ctypes.data)
    p = N.Params()
    L.fa2_default_params(C.byref(p))
    assert p.delta == 0.0
    p.delta = delta
    st = C.c_int(-1)
    ctx = L.fa2_create(C.byref(g), C.byref(p), C.byref(st))
    if ctx:
        L.fa2_destroy(ctx)
    return st.value


def test_create_checks_weights_before_the_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    for bad in (0.0, -2.0, np.nan, np.inf):
        assert _create_status([1.0, bad, 1.0], 1.0) == 1  # FA2_ERR_INVALID_ARGUMENT
        assert _create_status([1.0, bad, 1.0], 0.0) == 2  # weights unread: FA2_ERR_NO_DEVICE
    assert _create_status([1e30, 1.0, 1.0], 2.0) == 1     # w^delta past FLT_MAX
    assert _create_status([1.0, 1.0, 1.0], float("nan")) == 1
    assert _create_status([0.5, 2.0, 3.0], -1.0) == 2
    assert _create_status(None, 3.0) == 2


def _float64_restatement(g, xy, wd, linlog):
    f = np.zeros((g.n, 2))
    p = xy.astype(np.float64)
    for s, t, w in zip(g.sources[: g.m], g.targets[: g.m], wd.astype(np.float64)):
        d = p[t] - p[s]
        if linlog:
            r = np.hypot(*d)
            d = d * (np.log1p(r) / r)
        f[s] += w * d
        f[t] -= w * d
    return f


@pytest.mark.parametrize("linlog", [False, True])
def test_oracle_weighted_attraction(linlog):
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(400, 3, seed=2)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 2000, 2000, 3)
    plain = O.gravity_attraction(g, xy, 0.0, True, linlog=linlog)
    ones = np.ones(g.m, np.float32)
    assert np.array_equal(O.gravity_attraction(g, xy, 0.0, True, linlog, ones, 1.3), plain)
    w = np.random.default_rng(4).uniform(0.1, 10.0, g.m).astype(np.float32)
    for delta in (1.0, 0.5, -2.0):
        wd = O.edge_weight_powers(w, delta)
        got = O.gravity_attraction(g, xy, 0.0, True, linlog, w, delta)
        ref = _float64_restatement(g, xy, wd, linlog)
        assert np.sqrt(np.mean((got - ref) ** 2) / np.mean(ref ** 2)) < 1e-6, delta
    assert np.array_equal(O.gravity_attraction(g, xy, 0.0, True, linlog, w, 0.0), plain)


def test_engine_wants_one_weight_per_edge():
    from gpugraphlayout_b200 import Engine
    with pytest.raises(ValueError):
        Engine(3, [0, 1], [1, 2], weights=[1.0], delta=1.0)

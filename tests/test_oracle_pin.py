"""The oracle (oracle/fa2_oracle.c) against the reference's own code, run here:

* the reference's CUDA kernels (src/RPBHKernels.cu, src/RPFA2Kernels.cu)
  executed by the CPU SIMT emulator (oracle/_ref/libref_gpuemu.so), in
  CUDAForceAtlas2::doStep order: sort order, forces, positions and the
  adaptive speed must match bit for bit;
* the reference's host classes (oracle/_ref/libref_cpu.so): UGraph ids,
  degrees and adjacency order, initial positions, the gravity/attraction
  formulas and the speed rule.

These need the reference build (oracle/_ref); they are skipped without it.
"""
import os

import numpy as np
import pytest

from conftest import rel_rmse

O = pytest.importorskip("oracle.oracle")
pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


def _emu_vs_oracle(g, xy, k_r, k_g, sg, steps, tree_threads=32):
    fo = O.FA2(g, xy, k_r, k_g, sg)
    em = O.RefGPUEmu(g, xy, k_r, k_g, sg, tree_threads=tree_threads)
    try:
        for it in range(steps):
            fo.step()
            em.step()
            assert np.array_equal(fo.sortd, em.sortd), f"sortd differs at step {it}"
            assert np.array_equal(fo.f_ga, em.f_ga), f"gravity+attraction differ at step {it}"
            assert np.array_equal(fo.f_tot, em.f_tot), f"total force differs at step {it}"
            assert np.array_equal(fo.positions, em.positions()), f"positions differ at step {it}"
            assert fo.global_speed == em.global_speed
            assert fo.speed_efficiency == em.speed_efficiency
            assert fo.s.maxdepth == em.maxdepth
    finally:
        del em


@pytest.mark.parametrize("sg,k_r", [(True, 10.0), (False, 80.0)])
def test_oracle_matches_reference_kernels_ba(ba3k, sg, k_r):
    xy = O.random_positions(ba3k.n, 2000, 2000, 1234)
    _emu_vs_oracle(ba3k, xy, k_r, 1.0, sg, steps=4)


def test_oracle_matches_reference_kernels_clustered():
    """Positions in tight clusters: deep cells, many warp-vote descents."""
    from gpugraphlayout_b200 import synth
    s, t = synth.sbm_edges(1500, 6, 0.05, 0.002, 40, seed=3)
    g = O.Graph(s, t)
    rng = np.random.default_rng(5)
    centres = rng.uniform(-1000, 1000, size=(6, 2))
    xy = (centres[np.arange(g.n) % 6] + rng.normal(0, 3.0, size=(g.n, 2))).astype(np.float32)
    _emu_vs_oracle(g, xy, 2.0, 1.0, False, steps=3)


@pytest.mark.parametrize("n_pairs", [1, 2, 5])
def test_oracle_matches_reference_kernels_tiny(n_pairs):
    src = np.arange(n_pairs, dtype=np.uint32)
    dst = src + 1
    g = O.Graph(src, dst)
    xy = O.random_positions(g.n, 100, 100, 99)
    _emu_vs_oracle(g, xy, 1.0, 1.0, True, steps=3, tree_threads=1)


def _coincident_case():
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(400, 2, seed=2)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 500, 500, 4)
    xy[7] = xy[3]
    xy[11] = xy[3]
    xy[20] = xy[19]
    return g, xy


def test_reference_drops_bodies_after_a_coincidence():
    """Known reference defect, kept visible: after scaling a coincident body
    TreeBuildingKernel executes `break` (src/RPBHKernels.cu:277), which leaves
    the thread's insertion loop, so that thread inserts none of its remaining
    bodies and sortd is no longer a permutation.  The engine and the oracle
    follow the comment's intent instead ("start all over")."""
    g, xy = _coincident_case()
    em = O.RefGPUEmu(g, xy, 1.0, 1.0, True, tree_threads=1)
    try:
        em.step()
        assert len(np.unique(em.sortd)) < g.n
    finally:
        del em


def test_coincident_bodies_scaled_then_inserted():
    """The oracle scales each body that lands on an earlier one (by id) by .99
    and inserts it again.  The result is the reference's tree, sort order and
    repulsion on the scaled positions (which have no coincidences)."""
    g, xy = _coincident_case()
    t = O.Tree(xy, g.mass)
    assert t.n_perturbed == 4  # 7 once, 11 twice (onto 3, then onto 7), 20 once
    scaled = t.xy.reshape(-1, 2)
    assert np.array_equal(scaled[7], (xy[7].astype(np.float64) * .99).astype(np.float32))
    assert np.array_equal(scaled[11], (xy[11].astype(np.float64) * .99 * .99).astype(np.float32))
    assert np.array_equal(scaled[3], xy[3]) and np.array_equal(scaled[19], xy[19])
    rep, ovf, _ = t.repulsion(1.0)
    em = O.RefGPUEmu(g, scaled, 1.0, 1.0, True, tree_threads=1)
    try:
        em.step()
        assert np.array_equal(t.sort(), em.sortd)
        rep_ref = (em.f_tot - em.f_ga).reshape(-1, 2)
        assert rel_rmse(rep, rep_ref) < 1e-5  # difference of two rounded sums
    finally:
        del em


def deep_pair_positions():
    """Root box [-1024, 1024]^2; two bodies 2^-25 apart whose separating cell
    boundary (a multiple of 2^-24) is reached at level 35.  All cell centres
    are exact in float, so the split depth is certain."""
    return np.array([[-1024.0, -1024.0], [1024.0, 1024.0], [2.0 ** -25, 0.0],
                     [1.5 * 2.0 ** -24, 0.0]], np.float32)


def test_depth_overflow_disables_repulsion_like_reference():
    """Bodies that separate below level 32: the reference's force kernel then
    adds nothing at all (src/RPBHKernels.cu:595), in this and later steps."""
    g = O.Graph(np.array([0, 1, 2], np.uint32), np.array([1, 2, 3], np.uint32))
    xy = deep_pair_positions()
    fo = O.FA2(g, xy, 1.0, 1.0, True)
    em = O.RefGPUEmu(g, xy, 1.0, 1.0, True, tree_threads=1)
    try:
        fo.step()
        em.step()
        assert em.maxdepth > 32 and fo.s.depth_overflow == 1
        assert np.array_equal(fo.sortd, em.sortd)
        assert np.array_equal(fo.f_tot, em.f_tot)
        assert np.array_equal(fo.f_tot, fo.f_ga)  # no repulsion at all
    finally:
        del em


def test_cell_summaries_match_reference_kernels(ba3k):
    xy = O.random_positions(ba3k.n, 2000, 2000, 42)
    t = O.Tree(xy, ba3k.mass)
    em = O.RefGPUEmu(ba3k, xy, 1.0, 1.0, True, tree_threads=32)
    try:
        em.step()
        ref = em.cells()
        mine = t.cells()
        assert len(ref["mass"]) == len(mine["mass"])
        # same multiset of (mass, centre, count): cell numbering differs
        a = np.rec.fromarrays([mine["mass"], mine["cx"], mine["cy"], mine["count"]])
        b = np.rec.fromarrays([ref["mass"], ref["cx"], ref["cy"], ref["count"]])
        assert np.array_equal(np.sort(a), np.sort(b))
    finally:
        del em


# ----------------------------------------------------------- reference CPU --

EDGE_CASES = """# comment line
5 3
3 5
7 7
9 5
# another
5 3
1\t9
12 3
3 12
100 1
1 100
"""


def _write(tmp_path, text, name="g.txt"):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_ugraph_build_matches_reference_loader(tmp_path):
    path = _write(tmp_path, EDGE_CASES)
    rg = O.RefGraph(path)
    pairs = [tuple(map(int, l.split())) for l in EDGE_CASES.splitlines() if l and l[0] != "#"]
    s = np.array([p[0] for p in pairs], np.uint32)
    t = np.array([p[1] for p in pairs], np.uint32)
    og = O.Graph(s, t)
    assert og.n == rg.n and og.m == rg.m
    assert np.array_equal(og.node_map_r, rg.node_map_r())
    assert np.array_equal(og.degree, rg.degrees())
    off, adj = rg.adjacency()
    assert np.array_equal(adj.astype(np.int32), og.targets)
    assert np.array_equal(np.repeat(np.arange(rg.n), np.diff(off)).astype(np.int32), og.sources)


def test_ugraph_build_matches_reference_on_ba(tmp_path):
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(2000, 3, seed=9)
    # shuffle direction and order to exercise first-appearance ids
    rng = np.random.default_rng(0)
    perm = rng.permutation(len(s))
    flip = rng.random(len(s)) < 0.5
    s2, t2 = np.where(flip, t, s)[perm], np.where(flip, s, t)[perm]
    path = str(tmp_path / "ba.txt")
    synth.write_edgelist(path, s2, t2)
    rg = O.RefGraph(path)
    og = O.Graph(s2, t2)
    assert np.array_equal(og.node_map_r, rg.node_map_r())
    assert np.array_equal(og.degree, rg.degrees())
    off, adj = rg.adjacency()
    assert np.array_equal(adj.astype(np.int32), og.targets)


def test_initial_positions_match_reference(tmp_path):
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(500, 2, seed=1)
    path = str(tmp_path / "g.txt")
    synth.write_edgelist(path, s, t)
    rg = O.RefGraph(path)
    for w, h in ((10000.0, 10000.0), (2000.0, 2000.0), (20000.0, 20000.0)):
        ref = O.RefCPUFA2(rg, w, h, 1234, True, True, 1.0, 10.0)
        assert np.array_equal(ref.positions(), O.random_positions(rg.n, w, h, 1234))
        del ref


def test_gravity_attraction_formulas_match_reference_cpu(tmp_path):
    """CPUForceAtlas2's gravity and attraction (RPCPUForceAtlas2.cpp:55-83,
    104-124) are the same forces as the GPU kernels; summation order differs."""
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(1000, 3, seed=4)
    path = str(tmp_path / "g.txt")
    synth.write_edgelist(path, s, t)
    rg = O.RefGraph(path)
    og = O.Graph(s, t)
    for sg in (True, False):
        ref = O.RefCPUFA2(rg, 2000, 2000, 1234, True, sg, 1.0, 10.0)
        ga_ref, _ = ref.forces()
        ga = O.gravity_attraction(og, ref.positions(), 1.0, sg)
        assert rel_rmse(ga, ga_ref) < 1e-6
        del ref


def test_linlog_attraction_matches_reference_cpu(tmp_path):
    """The linear-log attraction of the reference's CPU path (use_linlog,
    RPCPUForceAtlas2.cpp:59-67; the GPU path ignores the flag) against the
    oracle's restatement, with gravity, on layouts whose edges span short and
    long distances; summation order differs."""
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(1000, 3, seed=5)
    path = str(tmp_path / "g.txt")
    synth.write_edgelist(path, s, t)
    rg = O.RefGraph(path)
    og = O.Graph(s, t)
    for sg, width in ((True, 2000.0), (False, 3.0)):
        ref = O.RefCPUFA2(rg, width, width, 1234, True, sg, 1.0, 10.0)
        ref.set_linlog(True)
        ga_ref, _ = ref.forces()
        ga = O.gravity_attraction(og, ref.positions(), 1.0, sg, linlog=True)
        lin = O.gravity_attraction(og, ref.positions(), 1.0, sg, linlog=False)
        assert rel_rmse(ga, ga_ref) < 1e-6
        assert rel_rmse(lin, ga_ref) > 1e-2  # the flag changes the forces
        del ref


def test_speed_rule_matches_reference_cpu(tmp_path):
    """The global-speed update (RPFA2Kernels.cu:177-219 = RPCPUForceAtlas2.cpp:144-197)."""
    g = O.Graph(np.array([0, 1], np.uint32), np.array([1, 2], np.uint32))
    path = _write(tmp_path, "0 1\n1 2\n")
    rg = O.RefGraph(path)
    ref = O.RefCPUFA2(rg, 100, 100, 1, True, True, 1.0, 1.0)
    L = O.ref_cpu()
    rng = np.random.default_rng(3)
    st = O.FA2(g, np.zeros((3, 2), np.float32), 1.0, 1.0, True)
    for _ in range(20):
        f = rng.normal(0, 50, size=(3, 2)).astype(np.float32)
        fp = rng.normal(0, 50, size=(3, 2)).astype(np.float32)
        L.refcpu_fa2_set_forces(ref._p, f.reshape(-1), fp.reshape(-1))
        L.refcpu_fa2_update_speeds(ref._p)
        # the oracle's rule from the same sums (sequential order for n = 3)
        swg = np.float32(0)
        etra = np.float32(0)
        for i in range(3):
            m = np.float32(g.mass[i])
            d = f[i] - fp[i]
            swg = np.float32(swg + m * np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1]))))
            d = f[i] + fp[i]
            etra = np.float32(etra + m * np.float32(np.sqrt(np.float32(d[0] * d[0] + d[1] * d[1])) / 2.0))
        sp = O._SpeedState(st.s.global_speed, st.s.speed_efficiency, 1.0, 10.0)
        O.lib().orc_speed_update(3, swg, etra, O.C.byref(sp))
        st.s.global_speed, st.s.speed_efficiency = sp.global_speed, sp.speed_efficiency
        assert sp.global_speed == pytest.approx(L.refcpu_fa2_global_speed(ref._p), rel=1e-6)
        assert sp.speed_efficiency == pytest.approx(L.refcpu_fa2_speed_efficiency(ref._p),
                                                    rel=1e-6)
    del ref

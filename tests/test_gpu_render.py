"""The GPU renderer (fa2_render_rgb, GraphLayout::writeToPNG) against the
oracle's restatement of the same pixel rules: identical images.  pngwriter,
which the reference draws with, is not in its sources, so the rules are the
engine's (coverage counts, discs of radius 3, Bresenham lines)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from test_host import _read_png

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,w,h", [(300, 200, 150), (20000, 640, 480), (40, 97, 61)])
def test_render_matches_oracle(n, w, h):
    from gpugraphlayout_b200 import render_rgb, synth
    from oracle import oracle as O
    s, t = synth.ba_edges(n, 3, seed=n)
    g = O.Graph(s, t)
    xy = O.random_positions(g.n, 1000, 700, 3)
    img = render_rgb(g.n, g.sources, g.targets, xy, w, h)
    ref = O.render(g.n, g.sources, g.targets, xy, w, h)
    assert np.array_equal(img, ref)
    # small graphs blend at opacity > 1: covered pixels are black
    if g.n < 10000:
        assert img.min() == 0


def test_cli_png_is_the_rendered_layout(tmp_path):
    """graph_viewer ... png w h writes the picture of the layout it computed:
    the same run written as bin and rendered gives the same image."""
    from gpugraphlayout_b200 import render_rgb, synth
    from oracle import oracle as O
    src, dst = synth.ba_edges(800, 2, seed=9)
    edges = str(tmp_path / "g.txt")
    synth.write_edgelist(edges, src, dst)
    exe = os.path.join(ROOT, "gpugraphlayout_b200", "graph_viewer")
    outs = {}
    for fmt in ("png", "bin"):
        d = tmp_path / fmt
        d.mkdir()
        args = [exe, "gpu", "20", "1", "sg", "10", "1", "approximate", edges, str(d), fmt]
        if fmt == "png":
            args += ["320", "240"]
        r = subprocess.run(args, capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        outs[fmt] = str(d / f"g.txt_20.{fmt}")
    png = _read_png(outs["png"])
    rec = np.fromfile(outs["bin"], dtype=np.dtype([("id", "<u4"), ("x", "<f4"), ("y", "<f4")]))
    g = O.Graph(src, dst)
    # the bin file lists UGraph ids with their edge-list ids: map back to UGraph order
    assert np.array_equal(rec["id"], g.node_map_r)
    xy = np.stack([rec["x"], rec["y"]], 1)
    assert np.array_equal(png, render_rgb(g.n, g.sources, g.targets, xy, 320, 240))

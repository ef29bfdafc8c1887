"""Drop-in check: the reference's own command-line source (src/graph_viewer.cpp),
compiled unchanged against this engine's headers (include/) and linked to
libfa2b200.so (oracle/_ref/graph_viewer_refsrc, built by `make -C oracle ref`),
writes exactly the layout this engine's graph_viewer writes."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

REFSRC_CLI = os.path.join(ROOT, "oracle", "_ref", "graph_viewer_refsrc")
CLI = os.path.join(ROOT, "gpugraphlayout_b200", "graph_viewer")


def test_reference_cli_source_builds_against_dropin_headers():
    if not os.path.exists(REFSRC_CLI):
        pytest.skip("oracle/_ref/graph_viewer_refsrc not built")
    r = subprocess.run([REFSRC_CLI], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Usage: graph_viewer" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("fmt,gravity", [("bin", "sg"), ("csv", "wg")])
def test_reference_cli_source_runs_on_engine(tmp_path, fmt, gravity):
    if not os.path.exists(REFSRC_CLI):
        pytest.skip("oracle/_ref/graph_viewer_refsrc not built")
    from gpugraphlayout_b200 import synth
    s, t = synth.ba_edges(3000, 3, seed=12)
    path = str(tmp_path / "g.txt")
    synth.write_edgelist(path, s, t)
    outs = []
    for exe, name in ((REFSRC_CLI, "ref"), (CLI, "ours")):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe, "gpu", "40", "2", gravity, "10", "1", "approximate", path, str(d),
                            fmt], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        outs.append(sorted(os.listdir(d)))
        outs.append([open(d / f, "rb").read() for f in sorted(os.listdir(d))])
    assert outs[0] == outs[2] == [f"g.txt_20.{fmt}", f"g.txt_40.{fmt}"]
    assert outs[1] == outs[3]

"""Host side, no GPU needed: the C-ABI library loads and exports what
include/fa2b200.h declares; the drop-in graph layer (C++ UGraph, layout
writers, random positions) gives the reference's results bit for bit; the
graph_viewer CLI checks its arguments as the reference does."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "fa2b200.h")
LIB = os.path.join(ROOT, "gpugraphlayout_b200", "libfa2b200.so")
CLI = os.path.join(ROOT, "gpugraphlayout_b200", "graph_viewer")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fa2_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    import ctypes
    lib = ctypes.CDLL(LIB)
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing
    from gpugraphlayout_b200 import _native
    assert sorted(_native.EXPORTS) == declared_symbols()


def test_status_strings_and_version():
    from gpugraphlayout_b200._native import lib
    L = lib()
    for s in range(9):
        assert L.fa2_status_string(s)
    assert b"sm_100a" in L.fa2_version()


def test_create_without_device_reports_status():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from gpugraphlayout_b200 import Engine, Fa2Error
    with pytest.raises(Fa2Error) as ei:
        Engine(3, [0, 1], [1, 2])
    assert ei.value.status == 2


EDGE_CASES = (
    "# comment\n5 3\n3 5\n7 7\n9 5\n#x\n5 3\n1\t9\n12 3\r\n3 12\n100 1\n1 100\n"
    "  4   8  \n8 4 trailing words\n+6 2\n"
)


def _pairs(text):
    out = []
    for line in text.splitlines():
        if not line or line[0] == "#":
            continue
        f = line.split()
        out.append((int(f[0]), int(f[1])))
    return np.array([p[0] for p in out], np.uint32), np.array([p[1] for p in out], np.uint32)


def test_ugraph_matches_oracle_on_edge_cases(tmp_path):
    from gpugraphlayout_b200 import UGraph
    from oracle import oracle as O
    p = tmp_path / "e.txt"
    p.write_text(EDGE_CASES)
    g = UGraph(str(p))
    s, t = _pairs(EDGE_CASES)
    og = O.Graph(s, t)
    assert g.num_nodes() == og.n and g.num_edges() == og.m
    assert np.array_equal(g.node_map_r, og.node_map_r)
    assert np.array_equal(g.degrees(), og.degree)
    es, et = g.edges()
    assert np.array_equal(es.astype(np.int32), og.sources)
    assert np.array_equal(et.astype(np.int32), og.targets)


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
                    reason="oracle/_ref not built")
@pytest.mark.parametrize("text", [EDGE_CASES, "1 2\n", "3 3\n", "# only comments\n"])
def test_ugraph_matches_reference_loader(tmp_path, text):
    from gpugraphlayout_b200 import UGraph
    from oracle import oracle as O
    p = tmp_path / "e.txt"
    p.write_text(text)
    g = UGraph(str(p))
    rg = O.RefGraph(str(p))
    assert g.num_nodes() == rg.n and g.num_edges() == rg.m
    assert np.array_equal(g.node_map_r, rg.node_map_r())
    assert np.array_equal(g.degrees(), rg.degrees())
    off, adj = rg.adjacency()
    es, et = g.edges()
    assert np.array_equal(et, adj)
    assert np.array_equal(es, np.repeat(np.arange(rg.n), np.diff(off)).astype(np.uint32))


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
                    reason="oracle/_ref not built")
def test_ugraph_matches_reference_on_rmat(tmp_path):
    from gpugraphlayout_b200 import UGraph, synth
    from oracle import oracle as O
    s, t = synth.rmat_edges(12, 40000, seed=1)
    rng = np.random.default_rng(2)
    perm = rng.permutation(len(s))
    flip = rng.random(len(s)) < 0.5
    s2 = np.where(flip, t, s)[perm]
    t2 = np.where(flip, s, t)[perm]
    # duplicates and self-loops in the file
    s2 = np.concatenate([s2, t2[:500], s2[:50]])
    t2 = np.concatenate([t2, s2[:500], s2[:50]])
    path = str(tmp_path / "r.txt")
    synth.write_edgelist(path, s2, t2)
    g = UGraph(path)
    rg = O.RefGraph(path)
    assert np.array_equal(g.node_map_r, rg.node_map_r())
    assert np.array_equal(g.degrees(), rg.degrees())
    off, adj = rg.adjacency()
    assert np.array_equal(g.edges()[1], adj)


def test_random_positions_match_oracle():
    from gpugraphlayout_b200 import random_positions
    from oracle import oracle as O
    for n, w in ((1, 10000.0), (1000, 2000.0), (5000, 2e4)):
        assert np.array_equal(random_positions(n, w, w, 1234), O.random_positions(n, w, w, 1234))


@pytest.mark.skipif(not __import__("oracle.oracle", fromlist=["x"]).ref_available(),
                    reason="oracle/_ref not built")
@pytest.mark.parametrize("binary", [0, 1])
def test_layout_writers_match_reference(tmp_path, binary):
    import gpugraphlayout_b200 as G
    from gpugraphlayout_b200 import synth
    from oracle import oracle as O
    s, t = synth.ba_edges(700, 2, seed=8)
    path = str(tmp_path / "g.txt")
    synth.write_edgelist(path, s + 3, t * 2 + 1)
    g = G.UGraph(path)
    rg = O.RefGraph(path)
    ref = O.RefCPUFA2(rg, 2000, 2000, 1234, True, True, 1.0, 1.0)
    rng = np.random.default_rng(0)
    xy = (rng.normal(0, 300, size=(g.num_nodes(), 2))).astype(np.float32)
    ref.set_positions(xy)
    a, b = str(tmp_path / "mine.out"), str(tmp_path / "ref.out")
    layout = G.GraphLayout(g)
    layout.xy[:] = xy
    (layout.writeToBin if binary else layout.writeToCSV)(a)
    ref.write(b, bool(binary))
    assert open(a, "rb").read() == open(b, "rb").read()
    with pytest.raises(G.Fa2Error):
        (layout.writeToBin if binary else layout.writeToCSV)(a)  # exists


def _cli(*args):
    return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)


def test_cli_argument_checks(tmp_path):
    r = _cli()
    assert r.returncode != 0 and "Usage: graph_viewer" in r.stderr
    p = tmp_path / "g.txt"
    p.write_text("1 2\n2 3\n")
    r = _cli("gpu", "5", "1", "sg", "1", "1", "exact", str(p), str(tmp_path), "bin")
    assert r.returncode != 0 and "requires Barnes-Hut" in r.stderr
    r = _cli("gpu", "5", "1", "sg", "1", "1", "approximate", str(tmp_path / "none.txt"),
             str(tmp_path), "bin")
    assert r.returncode != 0 and "No edgelist" in r.stderr
    r = _cli("gpu", "5", "1", "sg", "1", "1", "approximate", str(p), str(tmp_path / "nodir"), "bin")
    assert r.returncode != 0 and "No output folder" in r.stderr
    r = _cli("cpu", "5", "1", "sg", "1", "1", "approximate", str(p), str(tmp_path), "bin")
    assert r.returncode != 0 and "GPU" in r.stderr


def test_batch_create_checks_arguments_before_the_device():
    """fa2_batch_create refuses bad graphs and graphs past FA2_BATCH_MAX_NODES
    with a status, before it looks for a device."""
    import ctypes as C
    from gpugraphlayout_b200 import _native as N
    L = N.lib()
    p = N.Params()
    L.fa2_default_params(C.byref(p))
    s = np.array([0, 1], np.uint32)
    t = np.array([1, 1], np.uint32)  # a self-loop
    d = (N.GraphDesc * 1)()
    d[0] = N.GraphDesc(3, 2, s.ctypes.data, t.ctypes.data)
    st = C.c_int(-1)
    assert not L.fa2_batch_create(1, d, C.byref(p), C.byref(st))
    assert st.value == 1  # FA2_ERR_INVALID_ARGUMENT
    t2 = np.array([1, 2], np.uint32)
    d[0] = N.GraphDesc(N.FA2_BATCH_MAX_NODES + 1, 2, s.ctypes.data, t2.ctypes.data)
    assert not L.fa2_batch_create(1, d, C.byref(p), C.byref(st))
    assert st.value == 6  # FA2_ERR_TOO_LARGE


def _read_png(path):
    """Minimal PNG reader for 8-bit RGB, filter-0 files (what the engine writes):
    checks the signature and every chunk's CRC, returns an (h, w, 3) array."""
    import struct
    import zlib
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, w = 8, b"", None
    while pos < len(data):
        (n,) = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + n]
        (crc,) = struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])
        assert zlib.crc32(kind + body) == crc
        if kind == b"IHDR":
            w, h, depth, ctype, comp, filt, inter = struct.unpack(">IIBBBBB", body)
            assert (depth, ctype, comp, filt, inter) == (8, 2, 0, 0, 0)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(h, 1 + 3 * w)
    assert (raw[:, 0] == 0).all()
    return raw[:, 1:].reshape(h, w, 3)


def test_png_encoder_round_trip(tmp_path):
    from gpugraphlayout_b200 import write_png
    rng = np.random.default_rng(0)
    for h, w in ((5, 7), (1, 1), (300, 257)):  # the last needs several stored blocks
        img = rng.integers(0, 256, (h, w, 3), dtype=np.uint8)
        path = str(tmp_path / f"x{h}_{w}.png")
        write_png(img, path)
        assert np.array_equal(_read_png(path), img)

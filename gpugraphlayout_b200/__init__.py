"""B200-native ForceAtlas2 layout engine (drop-in for the GPU path of
govertb/GPUGraphLayout).

The engine is libfa2b200.so (C ABI in include/fa2b200.h, sm_100a kernels).
This module mirrors the reference's C++ interface for Python callers:

* ``UGraph(path)`` / ``UGraph.from_pairs(s, t)`` -- RPGraph::UGraph
* ``GraphLayout(graph, width=10000, height=10000)`` -- RPGraph::GraphLayout
* ``CUDAForceAtlas2(layout, use_barneshut, strong_gravity, gravity, scale)``
  -- RPGraph::CUDAForceAtlas2 (doStep, doSteps, sync_layout, setScale,
  setGravity, mass)
* ``Engine`` -- the C ABI context itself, with the test and measurement hooks
  (forces, body sort order, per-kernel timing).

Errors raise ``Fa2Error`` carrying the C status code; a missing library
raises at first use (there is no CPU fallback).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._native import Fa2Error, GraphDesc, Mlp, Params, Stats, check, lib

__all__ = ["Engine", "BatchEngine", "UGraph", "GraphLayout", "CUDAForceAtlas2", "Fa2Error", "kernel_names",
           "random_positions", "render_rgb", "write_png", "FarFieldMLP", "LearnSet"]


def _ptr(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else None


def kernel_names() -> list[str]:
    out, i = [], 0
    while True:
        s = lib().fa2_kernel_name(i)
        if s is None:
            return out
        out.append(s.decode())
        i += 1


def random_positions(n: int, width: float, height: float, seed: int = 1234) -> np.ndarray:
    """srandom(seed) + GraphLayout::randomizePositions: (n, 2) float32."""
    xy = np.zeros((max(n, 1), 2), np.float32)
    lib().fa2_random_positions(n, width, height, seed, _ptr(xy))
    return xy[:n].copy()


class Engine:
    """One fa2_ctx: a graph on the GPU with its ForceAtlas2 state.

    ``sources``/``targets`` list each undirected edge once over node ids
    0..num_nodes-1 (as UGraph.edges() returns them).  ``weights`` (optional,
    one positive weight per edge) with ``delta`` != 0 makes each edge attract
    with w**delta times the unweighted force (ForceAtlas2's edge weight
    influence; delta 0, the reference's default, ignores the weights)."""

    def __init__(self, num_nodes: int, sources, targets, *, strong_gravity: bool = False,
                 gravity: float = 1.0, scale: float = 1.0, theta: float = 1.0,
                 epssq: float = 0.05 * 0.05, device: int = 0, use_barneshut: bool = True,
                 linlog: bool = False, multipole: int = 1, weights=None, delta: float = 0.0):
        L = lib()
        self._src = np.ascontiguousarray(sources, np.uint32)
        self._dst = np.ascontiguousarray(targets, np.uint32)
        self._w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        if self._w is not None and len(self._w) != len(self._src):
            raise ValueError("one weight per edge")
        g = GraphDesc(num_nodes, len(self._src), _ptr(self._src), _ptr(self._dst),
                      _ptr(self._w))
        p = Params()
        L.fa2_default_params(C.byref(p))
        p.use_barneshut = int(use_barneshut)
        p.strong_gravity = int(strong_gravity)
        p.gravity, p.scale, p.theta, p.epssq, p.device = gravity, scale, theta, epssq, device
        p.linlog = int(linlog)
        p.multipole = int(multipole)
        p.delta = delta
        st = C.c_int(0)
        self._ctx = L.fa2_create(C.byref(g), C.byref(p), C.byref(st))
        check(st.value, "fa2_create")
        self.n = num_nodes

    def close(self):
        if getattr(self, "_ctx", None):
            lib().fa2_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- positions ---------------------------------------------------------
    def set_positions(self, xy) -> None:
        a = np.ascontiguousarray(xy, np.float32).reshape(self.n, 2)
        check(lib().fa2_set_positions(self._ctx, _ptr(a)), "fa2_set_positions")

    def get_positions(self, out: np.ndarray | None = None) -> np.ndarray:
        a = out if out is not None else np.zeros((self.n, 2), np.float32)
        check(lib().fa2_get_positions(self._ctx, _ptr(a)), "fa2_get_positions")
        return a

    def set_positions_ptr(self, host_ptr: int) -> None:
        """Upload from a raw host pointer (e.g. pinned memory)."""
        check(lib().fa2_set_positions(self._ctx, C.c_void_p(host_ptr)), "fa2_set_positions")

    def get_positions_ptr(self, host_ptr: int) -> None:
        check(lib().fa2_get_positions(self._ctx, C.c_void_p(host_ptr)), "fa2_get_positions")

    # -- stepping ----------------------------------------------------------
    def step(self, iters: int = 1) -> None:
        check(lib().fa2_step(self._ctx, iters), "fa2_step")

    def step_host(self, xy_in, iters: int, xy_out) -> None:
        """Positions in, iters steps, positions out, with one synchronisation
        (fa2_step_host).  xy_in and xy_out are float32 (n, 2) arrays (or None),
        or raw host pointers as ints (e.g. pinned memory)."""
        def arg(a, writable):
            if a is None or isinstance(a, int):
                return None if a is None else C.c_void_p(a)
            if not (isinstance(a, np.ndarray) and a.dtype == np.float32 and
                    a.flags["C_CONTIGUOUS"] and a.size == 2 * self.n and
                    (a.flags["WRITEABLE"] or not writable)):
                raise ValueError("positions: a C-contiguous float32 array of n x 2")
            return C.c_void_p(a.ctypes.data)
        check(lib().fa2_step_host(self._ctx, arg(xy_in, False), int(iters), arg(xy_out, True)),
              "fa2_step_host")

    def step_timed(self, iters: int, kernels: bool = True):
        """Runs iters steps; returns (device ms of the call, {kernel: mean ms per
        launch}).  kernels=False runs the steps without the per-kernel events
        (fa2_step's own graph) and returns an empty dict."""
        ms = C.c_float(0.0)
        if not kernels:
            check(lib().fa2_step_timed(self._ctx, iters, C.byref(ms), None, 0),
                  "fa2_step_timed")
            return ms.value, {}
        names = kernel_names()
        km = (C.c_float * len(names))()
        check(lib().fa2_step_timed(self._ctx, iters, C.byref(ms), km, len(names)),
              "fa2_step_timed")
        return ms.value, {nm: km[i] for i, nm in enumerate(names)}

    def set_force_params(self, scale: float, gravity: float) -> None:
        check(lib().fa2_set_force_params(self._ctx, scale, gravity), "fa2_set_force_params")

    def set_linlog(self, enable: bool) -> None:
        """Linear-log (True) or linear (False) attraction from the next step on."""
        check(lib().fa2_set_linlog(self._ctx, 1 if enable else 0), "fa2_set_linlog")

    def set_approximation(self, theta: float, multipole: int = 1) -> None:
        """Barnes-Hut opening parameter and far-field order from the next step
        on: multipole 1 treats accepted cells as point masses (the reference),
        2 adds each cell's quadrupole term."""
        check(lib().fa2_set_approximation(self._ctx, float(theta), int(multipole)),
              "fa2_set_approximation")

    def exact_repulsion(self, samples) -> np.ndarray:
        """Exact all-pairs repulsion (float64, computed on the GPU) of the
        nodes ``samples`` (reference ids) at the current positions, (k, 2)."""
        ids = np.ascontiguousarray(samples, np.uint32)
        out = np.zeros((len(ids), 2), np.float64)
        check(lib().fa2_exact_repulsion(self._ctx, len(ids), _ptr(ids), _ptr(out)),
              "fa2_exact_repulsion")
        return out

    def set_accuracy_guard(self, every: int, n_samples: int = 1024) -> None:
        """Every `every` steps, check the approximation against the FP64 sum
        on n_samples bodies and fall back to the reference walk (theta 1,
        monopole) when that is more accurate; 0 turns the guard off."""
        check(lib().fa2_set_accuracy_guard(self._ctx, int(every), int(n_samples)),
              "fa2_set_accuracy_guard")

    def accuracy_guard(self) -> dict:
        """The last check's relative RMSEs and the counts of checks and fallbacks."""
        ec, ep = C.c_double(0.0), C.c_double(0.0)
        ck, fb = C.c_int32(0), C.c_int32(0)
        check(lib().fa2_get_accuracy_guard(self._ctx, C.byref(ec), C.byref(ep), C.byref(ck),
                                           C.byref(fb)), "fa2_get_accuracy_guard")
        return {"err_current": ec.value, "err_plain": ep.value, "checks": ck.value,
                "fallbacks": fb.value}

    def set_learned_correction(self, mlp: "FarFieldMLP | None") -> None:
        """The learned far-field correction on top of the walk
        set_approximation selected, from the next step on; None turns it off."""
        check(lib().fa2_set_learned_correction(self._ctx, None if mlp is None else C.byref(mlp.c)),
              "fa2_set_learned_correction")

    def set_prevent_overlap(self, sizes) -> None:
        """ForceAtlas2's prevent_overlap with one size per node (reference
        ids), from the next step on; None turns it off."""
        if sizes is None:
            check(lib().fa2_set_prevent_overlap(self._ctx, None), "fa2_set_prevent_overlap")
            return
        sz = np.ascontiguousarray(sizes, np.float32).ravel()
        if len(sz) != self.n:
            raise Fa2Error(1, "set_prevent_overlap: one size per node")
        check(lib().fa2_set_prevent_overlap(self._ctx, _ptr(sz)), "fa2_set_prevent_overlap")

    def set_overlap(self, enable: bool) -> None:
        """Attraction beside the tree build (default) or alone before it."""
        check(lib().fa2_set_overlap(self._ctx, 1 if enable else 0), "fa2_set_overlap")

    # -- inspection ----------------------------------------------------------
    def forces(self):
        """(total, gravity + attraction) of the last step, each (n, 2)."""
        tot = np.zeros((self.n, 2), np.float32)
        ga = np.zeros((self.n, 2), np.float32)
        check(lib().fa2_get_forces(self._ctx, _ptr(tot), _ptr(ga)), "fa2_get_forces")
        return tot, ga

    def sort_order(self) -> np.ndarray:
        out = np.zeros(self.n, np.uint32)
        check(lib().fa2_get_sort_order(self._ctx, _ptr(out)), "fa2_get_sort_order")
        return out

    def stats(self) -> dict:
        s = Stats()
        check(lib().fa2_get_stats(self._ctx, C.byref(s)), "fa2_get_stats")
        return {f: getattr(s, f) for f, _ in Stats._fields_}

    def speed_state(self):
        gs, se = C.c_float(), C.c_float()
        fp = np.zeros((self.n, 2), np.float32)
        check(lib().fa2_get_speed_state(self._ctx, C.byref(gs), C.byref(se), _ptr(fp)),
              "fa2_get_speed_state")
        return gs.value, se.value, fp

    def set_speed_state(self, global_speed: float, speed_efficiency: float, f_prev=None):
        fp = None if f_prev is None else np.ascontiguousarray(f_prev, np.float32).reshape(self.n, 2)
        check(lib().fa2_set_speed_state(self._ctx, global_speed, speed_efficiency, _ptr(fp)),
              "fa2_set_speed_state")


class BatchEngine:
    """One fa2_batch: many independent graphs laid out together, each with the
    FA2 iteration of Engine and its own quadtree and speed state.

    ``graphs`` is a sequence of (num_nodes, sources, targets) with graph-local
    ids.  Positions and forces are (total nodes, 2) arrays, graph after graph."""

    def __init__(self, graphs, *, strong_gravity: bool = False, gravity: float = 1.0,
                 scale: float = 1.0, theta: float = 1.0, epssq: float = 0.05 * 0.05,
                 device: int = 0, linlog: bool = False):
        L = lib()
        self._keep = []
        descs = (GraphDesc * max(1, len(graphs)))()
        self.sizes = []
        for i, (n, s, t) in enumerate(graphs):
            s = np.ascontiguousarray(s, np.uint32)
            t = np.ascontiguousarray(t, np.uint32)
            self._keep += [s, t]
            descs[i] = GraphDesc(int(n), len(s), _ptr(s), _ptr(t))
            self.sizes.append(int(n))
        p = Params()
        L.fa2_default_params(C.byref(p))
        p.strong_gravity = int(strong_gravity)
        p.gravity, p.scale, p.theta, p.epssq, p.device = gravity, scale, theta, epssq, device
        p.linlog = int(linlog)
        st = C.c_int(0)
        self._b = L.fa2_batch_create(len(graphs), descs, C.byref(p), C.byref(st))
        check(st.value, "fa2_batch_create")
        self.num_graphs = len(graphs)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)]).astype(np.int64)
        self.n = int(self.offsets[-1])

    def close(self):
        if getattr(self, "_b", None):
            lib().fa2_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        self.close()

    def set_positions(self, xy) -> None:
        a = np.ascontiguousarray(xy, np.float32).reshape(self.n, 2)
        check(lib().fa2_batch_set_positions(self._b, _ptr(a)), "fa2_batch_set_positions")

    def get_positions(self) -> np.ndarray:
        out = np.zeros((self.n, 2), np.float32)
        check(lib().fa2_batch_get_positions(self._b, _ptr(out)), "fa2_batch_get_positions")
        return out

    def set_positions_ptr(self, host_ptr: int) -> None:
        """Upload from a raw host pointer (e.g. pinned memory), n x 2 floats."""
        check(lib().fa2_batch_set_positions(self._b, C.c_void_p(host_ptr)),
              "fa2_batch_set_positions")

    def get_positions_ptr(self, host_ptr: int) -> None:
        check(lib().fa2_batch_get_positions(self._b, C.c_void_p(host_ptr)),
              "fa2_batch_get_positions")

    def step(self, n_iters: int = 1) -> None:
        check(lib().fa2_batch_step(self._b, int(n_iters)), "fa2_batch_step")

    def step_timed(self, n_iters: int) -> float:
        ms = C.c_float(0.0)
        check(lib().fa2_batch_step_timed(self._b, int(n_iters), C.byref(ms)),
              "fa2_batch_step_timed")
        return ms.value

    def forces(self):
        tot = np.zeros((self.n, 2), np.float32)
        ga = np.zeros((self.n, 2), np.float32)
        check(lib().fa2_batch_get_forces(self._b, _ptr(tot), _ptr(ga)), "fa2_batch_get_forces")
        return tot, ga

    def sort_order(self) -> np.ndarray:
        out = np.zeros(max(1, self.n), np.uint32)
        check(lib().fa2_batch_get_sort_order(self._b, _ptr(out)), "fa2_batch_get_sort_order")
        return out[: self.n]

    def speeds(self):
        gs = np.zeros(max(1, self.num_graphs), np.float32)
        se = np.zeros(max(1, self.num_graphs), np.float32)
        check(lib().fa2_batch_get_speed(self._b, _ptr(gs), _ptr(se)), "fa2_batch_get_speed")
        return gs[: self.num_graphs], se[: self.num_graphs]

    def configure(self, split: int, small_threads: int = 256, large_threads: int = 1024) -> None:
        """Graphs of at most `split` nodes on CTAs of small_threads threads,
        the rest on CTAs of large_threads (split 0: one class)."""
        check(lib().fa2_batch_configure(self._b, int(split), int(small_threads),
                                        int(large_threads)), "fa2_batch_configure")

    def config(self) -> dict:
        sp, th, lt = C.c_uint32(0), C.c_int32(0), C.c_int32(0)
        check(lib().fa2_batch_get_config(self._b, C.byref(sp), C.byref(th), C.byref(lt)),
              "fa2_batch_get_config")
        return {"split": sp.value, "small_threads": th.value, "large_threads": lt.value}

    def autotune(self, iters: int = 2) -> dict:
        """Times the candidate configurations on this batch and keeps the
        fastest; the layout state is left as it was."""
        sp, th, lt, ms = C.c_uint32(0), C.c_int32(0), C.c_int32(0), C.c_float(0.0)
        check(lib().fa2_batch_autotune(self._b, int(iters), C.byref(sp), C.byref(th),
                                       C.byref(lt), C.byref(ms)), "fa2_batch_autotune")
        return {"split": sp.value, "small_threads": th.value, "large_threads": lt.value,
                "ms_per_iter": ms.value}

    def part(self, a, g: int):
        """Rows of graph g in a batch-ordered array."""
        return a[self.offsets[g]:self.offsets[g + 1]]


class UGraph:
    """RPGraph::UGraph: ids by first appearance, self-loops and repeated
    undirected edges dropped."""

    def __init__(self, edgelist_path: str | None = None, *, _handle=None):
        if _handle is None:
            st = C.c_int(0)
            _handle = lib().fa2_ugraph_load(str(edgelist_path).encode(), C.byref(st))
            check(st.value, f"UGraph({edgelist_path!r})")
        self._h = _handle
        self._deg = None

    @classmethod
    def from_pairs(cls, sources, targets) -> "UGraph":
        s = np.ascontiguousarray(sources, np.uint32)
        t = np.ascontiguousarray(targets, np.uint32)
        st = C.c_int(0)
        h = lib().fa2_ugraph_from_pairs(_ptr(s), _ptr(t), len(s), C.byref(st))
        check(st.value, "UGraph.from_pairs")
        return cls(_handle=h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().fa2_ugraph_free(self._h)
            self._h = None

    def num_nodes(self) -> int:
        return int(lib().fa2_ugraph_num_nodes(self._h))

    def num_edges(self) -> int:
        return int(lib().fa2_ugraph_num_edges(self._h))

    def degrees(self) -> np.ndarray:
        if self._deg is None:
            out = np.zeros(max(1, self.num_nodes()), np.uint32)
            check(lib().fa2_ugraph_degrees(self._h, _ptr(out)))
            self._deg = out[: self.num_nodes()]
        return self._deg

    def degree(self, nid: int) -> int:
        return int(self.degrees()[nid]) if nid < self.num_nodes() else 0

    in_degree = out_degree = degree

    @property
    def node_map_r(self) -> np.ndarray:
        out = np.zeros(max(1, self.num_nodes()), np.uint32)
        check(lib().fa2_ugraph_node_map_r(self._h, _ptr(out)))
        return out[: self.num_nodes()]

    def edges(self):
        m = self.num_edges()
        s = np.zeros(max(1, m), np.uint32)
        t = np.zeros(max(1, m), np.uint32)
        check(lib().fa2_ugraph_edges(self._h, _ptr(s), _ptr(t)))
        return s[:m], t[:m]

    def neighbors_with_geq_id(self, nid: int) -> list[int]:
        s, t = self.edges()
        return t[s == nid].tolist()


class GraphLayout:
    """RPGraph::GraphLayout: positions of a UGraph's nodes."""

    def __init__(self, graph: UGraph, width: float = 10000, height: float = 10000):
        self.graph = graph
        self.width, self.height = width, height
        self.xy = np.zeros((graph.num_nodes(), 2), np.float32)

    def randomizePositions(self, seed: int = 1234) -> None:
        """srandom(seed) as graph_viewer does at start-up, then the reference's draw."""
        self.xy[:] = random_positions(self.graph.num_nodes(), self.width, self.height, seed)

    def getX(self, n):
        return float(self.xy[n, 0])

    def getY(self, n):
        return float(self.xy[n, 1])

    def setX(self, n, v):
        self.xy[n, 0] = v

    def setY(self, n, v):
        self.xy[n, 1] = v

    def _write(self, path: str, binary: int):
        check(lib().fa2_write_layout(self.graph._h, _ptr(np.ascontiguousarray(self.xy)),
                                     str(path).encode(), binary), f"write {path}")

    def writeToCSV(self, path: str):
        self._write(path, 0)

    def writeToBin(self, path: str):
        self._write(path, 1)

    def writeToPNG(self, image_w: int, image_h: int, path: str):
        """The reference's picture of the layout, rendered on the GPU."""
        check(lib().fa2_write_png(self.graph._h, _ptr(np.ascontiguousarray(self.xy)),
                                  int(image_w), int(image_h), str(path).encode()),
              f"write {path}")


def render_rgb(num_nodes: int, sources, targets, xy, image_w: int, image_h: int,
               device: int = 0) -> np.ndarray:
    """GraphLayout::writeToPNG's picture as an (image_h, image_w, 3) uint8
    array, top row first, rendered on the GPU."""
    s = np.ascontiguousarray(sources, np.uint32)
    t = np.ascontiguousarray(targets, np.uint32)
    p = np.ascontiguousarray(xy, np.float32).reshape(-1, 2)
    out = np.zeros((image_h, image_w, 3), np.uint8)
    check(lib().fa2_render_rgb(int(num_nodes), len(s), _ptr(s), _ptr(t), _ptr(p), int(image_w),
                               int(image_h), int(device), _ptr(out)), "fa2_render_rgb")
    return out


def write_png(rgb, path: str) -> None:
    """An 8-bit RGB PNG of an (h, w, 3) uint8 array."""
    a = np.ascontiguousarray(rgb, np.uint8)
    check(lib().fa2_png_encode(_ptr(a), a.shape[1], a.shape[0], str(path).encode()),
          f"write {path}")


class FarFieldMLP:
    """fa2_mlp: the learned far-field correction's 12 -> 64 -> 64 -> 2 MLP
    (FP32 parameters; inference runs in BF16 with FP32 accumulation).  The
    arrays are views of the C struct, [out][in] like torch's nn.Linear."""

    NAMES = ("w1", "b1", "w2", "b2", "w3", "b3")
    SHAPES = {"w1": (64, 12), "b1": (64,), "w2": (64, 64), "b2": (64,), "w3": (2, 64), "b3": (2,)}

    def __init__(self, seed: int | None = 0):
        """nn.Linear's default initialisation from `seed`; None leaves zeros."""
        self.c = Mlp()
        if seed is not None:
            lib().fa2_mlp_init(C.byref(self.c), int(seed))

    def __getitem__(self, name: str) -> np.ndarray:
        return np.ctypeslib.as_array(getattr(self.c, name)).reshape(self.SHAPES[name])

    def __setitem__(self, name: str, value) -> None:
        self[name][...] = np.asarray(value, np.float32).reshape(self.SHAPES[name])

    def vector(self) -> np.ndarray:
        """All parameters as one float32 vector, in the struct's order."""
        return np.concatenate([self[n].ravel() for n in self.NAMES]).copy()

    @classmethod
    def from_vector(cls, v) -> "FarFieldMLP":
        m = cls(seed=None)
        v = np.asarray(v, np.float32).ravel()
        at = 0
        for n in cls.NAMES:
            k = int(np.prod(cls.SHAPES[n]))
            m[n] = v[at:at + k]
            at += k
        return m

    def forward(self, features, device: int = 0) -> np.ndarray:
        """The tensor-core inference kernel on (n, 12) features: (n, 2)."""
        x = np.ascontiguousarray(features, np.float32).reshape(-1, 12)
        out = np.zeros((len(x), 2), np.float32)
        check(lib().fa2_mlp_forward(int(device), C.byref(self.c), _ptr(x), len(x), _ptr(out)),
              "fa2_mlp_forward")
        return out

    def train_step(self, m: "FarFieldMLP", v: "FarFieldMLP", step: int, lr: float, features,
                   targets, weights, device: int = 0) -> float:
        """One Adam step of the training kernels on the given samples (in
        place, with Adam's moments m and v); returns the loss before it."""
        x = np.ascontiguousarray(features, np.float32).reshape(-1, 12)
        t = np.ascontiguousarray(targets, np.float32).reshape(-1, 2)
        w = np.ascontiguousarray(weights, np.float32).ravel()
        loss = C.c_float(0.0)
        check(lib().fa2_mlp_train_step(int(device), C.byref(self.c), C.byref(m.c), C.byref(v.c),
                                       int(step), float(lr), _ptr(x), _ptr(t), _ptr(w), len(x),
                                       C.byref(loss)), "fa2_mlp_train_step")
        return loss.value


class LearnSet:
    """fa2_learn_set: training samples of the learned correction in device
    memory, collected from an Engine's layouts (FP64 exact targets)."""

    def __init__(self, capacity: int, device: int = 0):
        st = C.c_int(0)
        self._h = lib().fa2_learn_set_create(int(device), int(capacity), C.byref(st))
        if not self._h:
            raise Fa2Error(st.value, "fa2_learn_set_create")

    def close(self):
        if getattr(self, "_h", None):
            lib().fa2_learn_set_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __len__(self) -> int:
        return int(lib().fa2_learn_set_size(self._h))

    def collect(self, engine: Engine, theta: float, multipole: int = 1) -> int:
        """Samples of the engine's current positions, walked at theta."""
        added = C.c_int64(0)
        check(lib().fa2_learn_collect(self._h, engine._ctx, float(theta), int(multipole),
                                      C.byref(added)), "fa2_learn_collect")
        return added.value

    def read(self, first: int = 0, count: int | None = None):
        """(features (k, 12), targets (k, 2), weights (k,)) of samples [first, first + k)."""
        count = len(self) - first if count is None else count
        f = np.zeros((count, 12), np.float32)
        t = np.zeros((count, 2), np.float32)
        w = np.zeros(count, np.float32)
        check(lib().fa2_learn_set_read(self._h, int(first), int(count), _ptr(f), _ptr(t),
                                       _ptr(w)), "fa2_learn_set_read")
        return f, t, w

    def fit(self, mlp: FarFieldMLP, steps: int, batch: int = 4096, lr: float = 2e-3,
            seed: int = 0) -> float:
        """Trains mlp in place with the training kernels; returns the last loss."""
        loss = C.c_float(0.0)
        check(lib().fa2_learn_fit(self._h, C.byref(mlp.c), int(steps), int(batch), float(lr),
                                  int(seed), C.byref(loss)), "fa2_learn_fit")
        return loss.value


class CUDAForceAtlas2:
    """RPGraph::CUDAForceAtlas2: the constructor randomizes the layout (as the
    reference's ForceAtlas2 constructor does) and uploads graph and positions."""

    def __init__(self, layout: GraphLayout, use_barneshut: bool, strong_gravity: bool,
                 gravity: float, scale: float, *, seed: int = 1234, device: int = 0):
        self.layout = layout
        self.k_r, self.k_g = scale, gravity
        self.strong_gravity = strong_gravity
        layout.randomizePositions(seed)
        s, t = layout.graph.edges()
        self.engine = Engine(layout.graph.num_nodes(), s, t, strong_gravity=strong_gravity,
                             gravity=gravity, scale=scale, device=device)
        self.engine.set_positions(layout.xy)
        self.iteration = 0
        # ForceAtlas2's public flags (src/RPForceAtlas2.hpp:44); the engine
        # honours use_linlog (linear-log attraction)
        self.use_linlog = False
        self.prevent_overlap = False

    def setScale(self, s: float):
        self.k_r = s

    def setGravity(self, g: float):
        self.k_g = g

    def mass(self, n: int) -> float:
        return self.layout.graph.degree(n) + 1.0

    def doStep(self):
        self.doSteps(1)

    def doSteps(self, n: int):
        self.engine.set_linlog(self.use_linlog)
        self.engine.set_force_params(self.k_r, self.k_g)
        self.engine.step(n)
        self.iteration += n

    def sync_layout(self):
        self.engine.get_positions(self.layout.xy)

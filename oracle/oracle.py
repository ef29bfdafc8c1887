"""ctypes bindings for the oracle (TEST INFRASTRUCTURE ONLY).

* ``liboracle.so``        -- the C restatement of the reference path (fa2_oracle.c)
* ``_ref/libref_cpu.so``  -- the reference's own host classes (UGraph,
  GraphLayout, CPUForceAtlas2), built from its sources by oracle/Makefile
* ``_ref/libref_gpuemu.so`` -- the reference's own CUDA kernels, run on the CPU
  by the SIMT emulator in oracle/ref

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  The engine in gpugraphlayout_b200/ never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")

_lib = None


class _SpeedState(C.Structure):
    _fields_ = [("global_speed", C.c_float), ("speed_efficiency", C.c_float),
                ("jitter_tolerance", C.c_float), ("k_s_max", C.c_float)]


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} is not built (run make -C oracle)")
        L = C.CDLL(path)
        L.orc_ugraph_build.restype = C.c_int64
        L.orc_ugraph_build.argtypes = [C.c_int64, _u32p, _u32p, _u32p, _u32p, _u32p,
                                       C.POINTER(C.c_int64)]
        L.orc_coo_order.argtypes = [C.c_int32, C.c_int64, _u32p, _u32p, _i32p, _i32p, _u32p]
        L.orc_random_positions.argtypes = [C.c_int32, C.c_float, C.c_float, C.c_uint32, _f32p]
        L.orc_gravity.argtypes = [C.c_int32, _f32p, _f32p, C.c_float, C.c_int32, _f32p, _f32p]
        L.orc_attraction.argtypes = [C.c_int64, _i32p, _i32p, _f32p, _f32p, _f32p]
        L.orc_attraction_linlog.argtypes = [C.c_int64, _i32p, _i32p, _f32p, _f32p, _f32p]
        L.orc_attraction_weighted.argtypes = [C.c_int64, _i32p, _i32p, _f32p, C.c_int32, _f32p,
                                              _f32p, _f32p]
        L.orc_tree_build.restype = C.c_void_p
        L.orc_tree_build.argtypes = [C.c_int32, _f32p, C.POINTER(C.c_int32)]
        L.orc_tree_free.argtypes = [C.c_void_p]
        L.orc_tree_maxdepth.restype = C.c_int32
        L.orc_tree_maxdepth.argtypes = [C.c_void_p]
        L.orc_tree_radius.restype = C.c_float
        L.orc_tree_radius.argtypes = [C.c_void_p]
        L.orc_tree_num_cells.restype = C.c_int32
        L.orc_tree_num_cells.argtypes = [C.c_void_p]
        L.orc_tree_root.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_tree_summarize.argtypes = [C.c_void_p, _f32p, _f32p]
        L.orc_tree_sort.argtypes = [C.c_void_p, _i32p]
        L.orc_tree_cells.argtypes = [C.c_void_p, _i32p, _f32p, _f32p, _f32p, _i32p]
        walk_args = [C.c_void_p, _f32p, _f32p, C.c_float, C.c_float, C.c_float, C.c_int32,
                     _i32p, _f32p, _f32p, C.POINTER(C.c_int64)]
        L.orc_tree_repulsion.restype = C.c_int32
        L.orc_tree_repulsion.argtypes = walk_args
        L.orc_tree_repulsion_quad.restype = C.c_int32
        L.orc_tree_repulsion_quad.argtypes = walk_args
        L.orc_tree_repulsion_overlap.restype = C.c_int32
        L.orc_tree_repulsion_overlap.argtypes = [C.c_void_p, _f32p, _f32p, _f32p, C.c_float,
                                                 C.c_float, C.c_float, C.c_int32, _i32p, _f32p,
                                                 _f32p, C.POINTER(C.c_int64)]
        L.orc_attraction_overlap.argtypes = [C.c_int64, _i32p, _i32p, _f32p, _f32p, _f32p, _f32p]
        L.orc_exact_repulsion_f64.argtypes = [C.c_int32, _f32p, _f32p, C.c_double, C.c_double,
                                              C.c_int32, _i32p, _f64p, _f64p]
        L.orc_fa2_step.restype = C.c_int32
        L.orc_fa2_step.argtypes = [C.c_void_p]
        L.orc_speed_update.argtypes = [C.c_int32, C.c_float, C.c_float, C.POINTER(_SpeedState)]
        _lib = L
    return _lib


# --------------------------------------------------------------------- graph --

class Graph:
    """The reference's UGraph applied to parsed (s, t) pairs (oracle restatement)."""

    def __init__(self, src, dst):
        src = np.ascontiguousarray(src, np.uint32)
        dst = np.ascontiguousarray(dst, np.uint32)
        n_pairs = len(src)
        node_map_r = np.zeros(max(1, 2 * n_pairs), np.uint32)
        lo = np.zeros(max(1, n_pairs), np.uint32)
        hi = np.zeros(max(1, n_pairs), np.uint32)
        ne = C.c_int64(0)
        n = lib().orc_ugraph_build(n_pairs, src, dst, node_map_r, lo, hi, C.byref(ne))
        if n < 0:
            raise MemoryError("orc_ugraph_build")
        self.n = int(n)
        self.m = int(ne.value)
        self.node_map_r = node_map_r[: self.n].copy()
        self.e_lo = lo[: self.m].copy()
        self.e_hi = hi[: self.m].copy()
        self.sources = np.zeros(max(1, self.m), np.int32)
        self.targets = np.zeros(max(1, self.m), np.int32)
        self.degree = np.zeros(max(1, self.n), np.uint32)
        lib().orc_coo_order(self.n, self.m, self.e_lo if self.m else lo, self.e_hi if self.m else hi,
                            self.sources, self.targets, self.degree)
        self.sources = self.sources[: self.m]
        self.targets = self.targets[: self.m]
        self.degree = self.degree[: self.n]
        self.mass = (self.degree.astype(np.float32) + np.float32(1.0))


def random_positions(n: int, width: float, height: float, seed: int = 1234) -> np.ndarray:
    xy = np.zeros(2 * max(n, 1), np.float32)
    lib().orc_random_positions(n, width, height, seed, xy)
    return xy[: 2 * n].reshape(n, 2).copy()


# ---------------------------------------------------------------- pieces --

def edge_weight_powers(weights, delta: float) -> np.ndarray:
    """w**delta per edge, from float32 weights in double, rounded once to float32."""
    w = np.ascontiguousarray(weights, np.float32).astype(np.float64)
    return np.power(w, float(delta)).astype(np.float32)


def gravity_attraction(g: Graph, xy: np.ndarray, k_g: float, strong: bool, linlog: bool = False,
                       weights=None, delta: float = 0.0, sizes=None):
    """Gravity plus attraction per node; with weights and delta != 0, each edge's
    attraction times w**delta (orc_attraction_weighted); with sizes, the
    prevent_overlap attraction (orc_attraction_overlap)."""
    n = g.n
    fx = np.zeros(n, np.float32)
    fy = np.zeros(n, np.float32)
    p = np.ascontiguousarray(xy, np.float32).reshape(-1)
    lib().orc_gravity(n, p, g.mass, k_g, int(strong), fx, fy)
    if sizes is not None:
        lib().orc_attraction_overlap(g.m, g.sources, g.targets,
                                     np.ascontiguousarray(sizes, np.float32), p, fx, fy)
    elif weights is not None and delta != 0.0:
        wd = edge_weight_powers(weights, delta)
        lib().orc_attraction_weighted(g.m, g.sources, g.targets, wd, int(linlog), p, fx, fy)
    else:
        attract = lib().orc_attraction_linlog if linlog else lib().orc_attraction
        attract(g.m, g.sources, g.targets, p, fx, fy)
    return np.stack([fx, fy], 1)


class Tree:
    """The reference quadtree (sequential TreeBuildingKernel) of positions xy.
    Like the reference, building may scale coincident bodies by .99; the
    possibly changed positions are in .xy."""

    def __init__(self, xy: np.ndarray, mass: np.ndarray):
        self.xy = np.ascontiguousarray(xy, np.float32).reshape(-1).copy()
        self.mass = np.ascontiguousarray(mass, np.float32)
        self.n = len(self.mass)
        pert = C.c_int32(0)
        self._t = lib().orc_tree_build(self.n, self.xy, C.byref(pert))
        if not self._t:
            raise MemoryError("orc_tree_build")
        self.n_perturbed = pert.value
        lib().orc_tree_summarize(self._t, self.xy, self.mass)

    def __del__(self):
        if getattr(self, "_t", None):
            lib().orc_tree_free(self._t)
            self._t = None

    @property
    def maxdepth(self):
        return lib().orc_tree_maxdepth(self._t)

    @property
    def radius(self):
        return lib().orc_tree_radius(self._t)

    @property
    def root(self):
        x, y = C.c_float(), C.c_float()
        lib().orc_tree_root(self._t, C.byref(x), C.byref(y))
        return x.value, y.value

    def sort(self) -> np.ndarray:
        out = np.zeros(max(1, self.n), np.int32)
        lib().orc_tree_sort(self._t, out)
        return out[: self.n]

    def cells(self):
        nc = lib().orc_tree_num_cells(self._t)
        level = np.zeros(nc, np.int32)
        mass = np.zeros(nc, np.float32)
        cx = np.zeros(nc, np.float32)
        cy = np.zeros(nc, np.float32)
        count = np.zeros(nc, np.int32)
        lib().orc_tree_cells(self._t, level, mass, cx, cy, count)
        return dict(level=level, mass=mass, cx=cx, cy=cy, count=count)

    def repulsion(self, k_r: float, itolsq: float = 1.0, epssq: float = 0.05 * 0.05,
                  group: int = 32, multipole: int = 1, sizes=None):
        fx = np.zeros(self.n, np.float32)
        fy = np.zeros(self.n, np.float32)
        visits = C.c_int64(0)
        if sizes is not None:
            sz = np.ascontiguousarray(sizes, np.float32)
            ovf = lib().orc_tree_repulsion_overlap(self._t, self.xy, self.mass, sz, k_r, itolsq,
                                                   np.float32(epssq), group, self.sort(), fx,
                                                   fy, C.byref(visits))
            return np.stack([fx, fy], 1), bool(ovf), visits.value
        walk = lib().orc_tree_repulsion_quad if multipole >= 2 else lib().orc_tree_repulsion
        ovf = walk(self._t, self.xy, self.mass, k_r, itolsq, np.float32(epssq),
                   group, self.sort(), fx, fy, C.byref(visits))
        return np.stack([fx, fy], 1), bool(ovf), visits.value


def exact_repulsion_f64(xy: np.ndarray, mass: np.ndarray, k_r: float, samples,
                        eps: float = float(np.float32(0.05 * 0.05))) -> np.ndarray:
    p = np.ascontiguousarray(xy, np.float32).reshape(-1)
    m = np.ascontiguousarray(mass, np.float32)
    s = np.ascontiguousarray(samples, np.int32)
    fx = np.zeros(len(s), np.float64)
    fy = np.zeros(len(s), np.float64)
    lib().orc_exact_repulsion_f64(len(m), p, m, k_r, eps, len(s), s, fx, fy)
    return np.stack([fx, fy], 1)


# ---------------------------------------------------------------- stepping --

class _OrcFa2(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("m", C.c_int64),
        ("sources", C.c_void_p), ("targets", C.c_void_p),
        ("xy", C.c_void_p), ("mass", C.c_void_p),
        ("fx", C.c_void_p), ("fy", C.c_void_p), ("fxp", C.c_void_p), ("fyp", C.c_void_p),
        ("k_r", C.c_float), ("k_g", C.c_float), ("strong_gravity", C.c_int32),
        ("itolsq", C.c_float), ("epssq", C.c_float), ("group", C.c_int32),
        ("speed_threads", C.c_int32),
        ("global_speed", C.c_float), ("speed_efficiency", C.c_float),
        ("jitter_tolerance", C.c_float), ("k_s_max", C.c_float),
        ("sortd_out", C.c_void_p), ("f_ga_out", C.c_void_p), ("f_tot_out", C.c_void_p),
        ("maxdepth", C.c_int32), ("n_perturbed", C.c_int32), ("depth_overflow", C.c_int32),
        ("swg_sum", C.c_float), ("etra_sum", C.c_float), ("linlog", C.c_int32),
        ("sizes", C.c_void_p),
    ]


class FA2:
    """The reference GPU path's iteration (CUDAForceAtlas2::doStep) restated on the CPU."""

    def __init__(self, g: Graph, xy: np.ndarray, k_r: float, k_g: float, strong_gravity: bool,
                 linlog: bool = False, sizes=None):
        self.g = g
        n = g.n
        self.xy = np.ascontiguousarray(xy, np.float32).reshape(-1).copy()
        self.fx = np.zeros(n, np.float32)
        self.fy = np.zeros(n, np.float32)
        self.fxp = np.zeros(n, np.float32)
        self.fyp = np.zeros(n, np.float32)
        self.sortd = np.zeros(n, np.int32)
        self.f_ga = np.zeros(2 * n, np.float32)
        self.f_tot = np.zeros(2 * n, np.float32)
        s = _OrcFa2()
        s.n, s.m = n, g.m
        s.sources, s.targets = g.sources.ctypes.data, g.targets.ctypes.data
        s.xy, s.mass = self.xy.ctypes.data, g.mass.ctypes.data
        s.fx, s.fy, s.fxp, s.fyp = (a.ctypes.data for a in (self.fx, self.fy, self.fxp, self.fyp))
        s.k_r, s.k_g, s.strong_gravity = k_r, k_g, int(strong_gravity)
        s.itolsq, s.epssq = 1.0, float(np.float32(0.05 * 0.05))
        s.group, s.speed_threads = 32, 512
        s.global_speed, s.speed_efficiency, s.jitter_tolerance, s.k_s_max = 1.0, 1.0, 1.0, 10.0
        s.sortd_out = self.sortd.ctypes.data
        s.f_ga_out = self.f_ga.ctypes.data
        s.f_tot_out = self.f_tot.ctypes.data
        s.maxdepth = 1
        s.linlog = int(linlog)
        # prevent_overlap with these node sizes (None: off)
        self._sizes = None if sizes is None else np.ascontiguousarray(sizes, np.float32)
        s.sizes = None if self._sizes is None else self._sizes.ctypes.data
        self.s = s

    def step(self, iters: int = 1):
        for _ in range(iters):
            if lib().orc_fa2_step(C.byref(self.s)) != 0:
                raise MemoryError("orc_fa2_step")

    @property
    def positions(self):
        return self.xy.reshape(-1, 2).copy()

    @property
    def global_speed(self):
        return self.s.global_speed

    @property
    def speed_efficiency(self):
        return self.s.speed_efficiency


# ------------------------------------------------------- reference libraries --

def ref_available() -> bool:
    return all(os.path.exists(os.path.join(HERE, "_ref", f))
               for f in ("libref_cpu.so", "libref_gpuemu.so"))


_ref_cpu = None
_ref_gpu = None


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        L = C.CDLL(os.path.join(HERE, "_ref", "libref_cpu.so"))
        vp = C.c_void_p
        L.refcpu_load.restype = vp
        L.refcpu_load.argtypes = [C.c_char_p]
        L.refcpu_graph_from_arrays.restype = vp
        L.refcpu_graph_from_arrays.argtypes = [C.c_uint32, _u32p, C.c_uint64, _u32p, _u32p]
        L.refcpu_free_graph.argtypes = [vp]
        L.refcpu_num_nodes.restype = C.c_uint32
        L.refcpu_num_nodes.argtypes = [vp]
        L.refcpu_num_edges.restype = C.c_uint32
        L.refcpu_num_edges.argtypes = [vp]
        L.refcpu_node_map_r.argtypes = [vp, _u32p]
        L.refcpu_degrees.argtypes = [vp, _u32p]
        L.refcpu_adjacency.argtypes = [vp, _u32p, _u32p]
        L.refcpu_fa2_create.restype = vp
        L.refcpu_fa2_create.argtypes = [vp, C.c_float, C.c_float, C.c_uint32, C.c_int, C.c_int,
                                        C.c_float, C.c_float]
        L.refcpu_fa2_destroy.argtypes = [vp]
        L.refcpu_fa2_positions.argtypes = [vp, _f32p]
        L.refcpu_fa2_set_positions.argtypes = [vp, _f32p]
        L.refcpu_fa2_step.argtypes = [vp, C.c_int]
        L.refcpu_fa2_global_speed.restype = C.c_float
        L.refcpu_fa2_global_speed.argtypes = [vp]
        L.refcpu_fa2_speed_efficiency.restype = C.c_float
        L.refcpu_fa2_speed_efficiency.argtypes = [vp]
        L.refcpu_fa2_forces.argtypes = [vp, _f32p, _f32p]
        L.refcpu_fa2_set_forces.argtypes = [vp, _f32p, _f32p]
        L.refcpu_fa2_update_speeds.argtypes = [vp]
        L.refcpu_fa2_set_linlog.argtypes = [vp, C.c_int]
        L.refcpu_fa2_write.argtypes = [vp, C.c_char_p, C.c_int]
        _ref_cpu = L
    return _ref_cpu


class RefGraph:
    """The reference's RPGraph::UGraph loaded from an edge-list file."""

    def __init__(self, path: str | None = None, *, graph: "Graph | None" = None):
        """From an edge-list file (the reference's loader), or from an oracle
        Graph (filled into the reference's members without re-reading a file)."""
        L = ref_cpu()
        if graph is not None:
            self._g = L.refcpu_graph_from_arrays(graph.n, graph.node_map_r, graph.m,
                                                 graph.e_lo, graph.e_hi)
        else:
            self._g = L.refcpu_load(path.encode())
        self.n = L.refcpu_num_nodes(self._g)
        self.m = L.refcpu_num_edges(self._g)

    def node_map_r(self):
        out = np.zeros(max(1, self.n), np.uint32)
        ref_cpu().refcpu_node_map_r(self._g, out)
        return out[: self.n]

    def degrees(self):
        out = np.zeros(max(1, self.n), np.uint32)
        ref_cpu().refcpu_degrees(self._g, out)
        return out[: self.n]

    def adjacency(self):
        off = np.zeros(self.n + 1, np.uint32)
        adj = np.zeros(max(1, self.m), np.uint32)
        ref_cpu().refcpu_adjacency(self._g, off, adj)
        return off, adj[: self.m]

    def __del__(self):
        if getattr(self, "_g", None):
            ref_cpu().refcpu_free_graph(self._g)
            self._g = None


class RefCPUFA2:
    """The reference's CPUForceAtlas2 on a RefGraph (srandom(seed) first)."""

    def __init__(self, g: RefGraph, width: float, height: float, seed: int, use_bh: bool,
                 strong_gravity: bool, gravity: float, scale: float):
        self.g = g
        self._p = ref_cpu().refcpu_fa2_create(g._g, width, height, seed, int(use_bh),
                                              int(strong_gravity), gravity, scale)

    def positions(self):
        out = np.zeros(2 * max(1, self.g.n), np.float32)
        ref_cpu().refcpu_fa2_positions(self._p, out)
        return out[: 2 * self.g.n].reshape(-1, 2).copy()

    def set_positions(self, xy):
        ref_cpu().refcpu_fa2_set_positions(self._p, np.ascontiguousarray(xy, np.float32).reshape(-1))

    def step(self, iters: int = 1):
        ref_cpu().refcpu_fa2_step(self._p, iters)

    def set_linlog(self, on: bool):
        ref_cpu().refcpu_fa2_set_linlog(self._p, int(on))

    def forces(self):
        n = self.g.n
        ga = np.zeros(2 * max(1, n), np.float32)
        rep = np.zeros(2 * max(1, n), np.float32)
        ref_cpu().refcpu_fa2_forces(self._p, ga, rep)
        return ga[: 2 * n].reshape(-1, 2), rep[: 2 * n].reshape(-1, 2)

    @property
    def global_speed(self):
        return ref_cpu().refcpu_fa2_global_speed(self._p)

    def write(self, path: str, binary: bool):
        ref_cpu().refcpu_fa2_write(self._p, path.encode(), int(binary))

    def __del__(self):
        if getattr(self, "_p", None):
            ref_cpu().refcpu_fa2_destroy(self._p)
            self._p = None


def ref_gpuemu():
    global _ref_gpu
    if _ref_gpu is None:
        L = C.CDLL(os.path.join(HERE, "_ref", "libref_gpuemu.so"))
        vp = C.c_void_p
        L.refgpu_create.restype = vp
        L.refgpu_create.argtypes = [C.c_int, C.c_int, _f32p, _f32p, _i32p, _i32p, C.c_int,
                                    C.c_float, C.c_float, C.c_int]
        L.refgpu_destroy.argtypes = [vp]
        L.refgpu_step.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p]
        L.refgpu_get_positions.argtypes = [vp, _f32p]
        L.refgpu_set_positions.argtypes = [vp, _f32p]
        for name in ("refgpu_global_speed", "refgpu_speed_efficiency", "refgpu_radius"):
            getattr(L, name).restype = C.c_float
            getattr(L, name).argtypes = []
        for name in ("refgpu_maxdepth", "refgpu_bottom"):
            getattr(L, name).restype = C.c_int
            getattr(L, name).argtypes = []
        L.refgpu_cells.restype = C.c_int
        L.refgpu_cells.argtypes = [vp, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _ref_gpu = L
    return _ref_gpu


class RefGPUEmu:
    """The reference's GPU kernels in doStep order, run by the CPU SIMT emulator.
    Only one instance may be alive at a time (the kernels keep file-static state,
    as on a GPU)."""

    def __init__(self, g: Graph, xy, k_r: float, k_g: float, strong_gravity: bool,
                 tree_threads: int = 1):
        self.n = g.n
        p = np.ascontiguousarray(xy, np.float32).reshape(-1)
        self._src = np.ascontiguousarray(g.sources, np.int32)
        self._dst = np.ascontiguousarray(g.targets, np.int32)
        self._h = ref_gpuemu().refgpu_create(g.n, g.m, p, np.ascontiguousarray(g.mass, np.float32),
                                             self._src if g.m else np.zeros(1, np.int32),
                                             self._dst if g.m else np.zeros(1, np.int32),
                                             int(strong_gravity), k_g, k_r, tree_threads)

    def step(self):
        n = self.n
        self.f_ga = np.zeros(2 * n, np.float32)
        self.f_tot = np.zeros(2 * n, np.float32)
        self.sortd = np.zeros(n, np.int32)
        ref_gpuemu().refgpu_step(self._h, self.f_ga.ctypes.data, self.f_tot.ctypes.data,
                                 self.sortd.ctypes.data)

    def positions(self):
        out = np.zeros(2 * self.n, np.float32)
        ref_gpuemu().refgpu_get_positions(self._h, out)
        return out.reshape(-1, 2)

    def cells(self):
        L = ref_gpuemu()
        nc = L.refgpu_cells(self._h, None, None, None, None)
        mass = np.zeros(nc, np.float32)
        cx = np.zeros(nc, np.float32)
        cy = np.zeros(nc, np.float32)
        count = np.zeros(nc, np.int32)
        L.refgpu_cells(self._h, mass.ctypes.data, cx.ctypes.data, cy.ctypes.data, count.ctypes.data)
        return dict(mass=mass, cx=cx, cy=cy, count=count)

    @property
    def global_speed(self):
        return ref_gpuemu().refgpu_global_speed()

    @property
    def speed_efficiency(self):
        return ref_gpuemu().refgpu_speed_efficiency()

    @property
    def maxdepth(self):
        return ref_gpuemu().refgpu_maxdepth()

    @property
    def radius(self):
        return ref_gpuemu().refgpu_radius()

    def __del__(self):
        if getattr(self, "_h", None):
            ref_gpuemu().refgpu_destroy(self._h)
            self._h = None


# -------------------------------------------------------------- rendering --

def render(n: int, sources, targets, xy, image_w: int, image_h: int) -> np.ndarray:
    """The layout picture of GraphLayout::writeToPNG (src/RPGraphLayout.cpp:
    170-207) restated with the pixel rules of the engine's renderer: frame in
    the reference's float/double arithmetic, positions truncated to int,
    1-based pixels with y up; discs of radius 3; Bresenham lines; each pixel
    white times (1 - a_node)^discs (1 - a_edge)^lines, black once a plot with
    opacity >= 1 covers it.  Returns (h, w, 3) uint8, top row first."""
    f32 = np.float32
    xy = np.asarray(xy, f32).reshape(-1, 2)
    s = np.asarray(sources, np.int64)
    t = np.asarray(targets, np.int64)
    mnx, mxx = f32(xy[:, 0].min()), f32(xy[:, 0].max())
    mny, mxy = f32(xy[:, 1].min()), f32(xy[:, 1].max())
    x_range, y_range = f32(mxx - mnx), f32(mxy - mny)
    x_center = f32(np.float64(mnx) + np.float64(x_range) / 2.0)
    y_center = f32(np.float64(mny) + np.float64(y_range) / 2.0)
    minx = f32(np.float64(x_center) - np.float64(x_range) / 2.0)
    miny = f32(np.float64(y_center) - np.float64(y_range) / 2.0)
    with np.errstate(divide="ignore"):
        xs, ys = f32(f32(image_w) / x_range), f32(f32(image_h) / y_range)
    a_node = f32(10000.0 / n)
    a_edge = f32(100000.0 / len(s)) if len(s) else f32(np.inf)
    px = np.trunc(f32(xy[:, 0] - minx) * xs).astype(np.int64)
    py = np.trunc(f32(xy[:, 1] - miny) * ys).astype(np.int64)
    cn = np.zeros((image_h, image_w), np.int64)
    ce = np.zeros((image_h, image_w), np.int64)

    def plot(cnt, x, y):
        ok = (x >= 1) & (x <= image_w) & (y >= 1) & (y <= image_h)
        np.add.at(cnt, (image_h - y[ok], x[ok] - 1), 1)

    for dy in range(-3, 4):
        for dx in range(-3, 4):
            if dx * dx + dy * dy <= 9:
                plot(cn, px + dx, py + dy)
    if len(s):
        x1, y1, x2, y2 = px[s], py[s], px[t], py[t]
        ax, ay = np.abs(x2 - x1), np.abs(y2 - y1)
        sx, sy = np.where(x2 >= x1, 1, -1), np.where(y2 >= y1, 1, -1)
        xmajor = ax >= ay
        D, d = np.where(xmajor, ax, ay), np.where(xmajor, ay, ax)
        steps = D + 1
        e = np.repeat(np.arange(len(s)), steps)
        tt = np.arange(steps.sum()) - np.repeat(np.cumsum(steps) - steps, steps)
        De, de = D[e], d[e]
        mi = np.where(De > 0, (2 * tt * de + De) // np.maximum(2 * De, 1), 0)
        x = np.where(xmajor[e], x1[e] + sx[e] * tt, x1[e] + sx[e] * mi)
        y = np.where(xmajor[e], y1[e] + sy[e] * mi, y1[e] + sy[e] * tt)
        plot(ce, x, y)
    with np.errstate(over="ignore", invalid="ignore"):
        v = np.power(1.0 - np.float64(a_node), cn) * np.power(1.0 - np.float64(a_edge), ce)
    v = np.where(((cn > 0) & (a_node >= 1)) | ((ce > 0) & (a_edge >= 1)), 0.0, v)
    c = np.minimum(255.0, np.floor(v * 255.0 + 0.5)).astype(np.uint8)
    return np.repeat(c[:, :, None], 3, axis=2)

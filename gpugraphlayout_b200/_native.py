"""ctypes declarations of libfa2b200.so (include/fa2b200.h).

The library is built in-tree by ``make -C gpugraphlayout_b200`` (or
``__graft_entry__.build()``).  Importing this module without it raises: there
is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfa2b200.so")

# Exported names declared in include/fa2b200.h.
EXPORTS = (
    "fa2_default_params", "fa2_create", "fa2_destroy", "fa2_set_positions",
    "fa2_get_positions", "fa2_step", "fa2_step_host", "fa2_step_timed", "fa2_kernel_name",
    "fa2_get_stats", "fa2_get_forces", "fa2_get_sort_order", "fa2_set_speed_state",
    "fa2_get_speed_state", "fa2_set_force_params", "fa2_set_linlog", "fa2_set_overlap",
    "fa2_set_approximation", "fa2_exact_repulsion", "fa2_last_cuda_error",
    "fa2_set_accuracy_guard", "fa2_get_accuracy_guard",
    "fa2_batch_create", "fa2_batch_destroy", "fa2_batch_set_positions", "fa2_batch_get_positions",
    "fa2_batch_step", "fa2_batch_step_timed", "fa2_batch_get_forces", "fa2_batch_get_sort_order",
    "fa2_batch_configure", "fa2_batch_get_config", "fa2_batch_autotune",
    "fa2_batch_get_speed", "fa2_render_rgb", "fa2_png_encode", "fa2_write_png", "fa2_repulsion_noalloc", "fa2_ugraph_load",
    "fa2_ugraph_from_pairs", "fa2_ugraph_free", "fa2_ugraph_num_nodes",
    "fa2_ugraph_num_edges", "fa2_ugraph_node_map_r", "fa2_ugraph_degrees",
    "fa2_ugraph_edges", "fa2_random_positions", "fa2_write_layout",
    "fa2_status_string", "fa2_version",
    "fa2_mlp_init", "fa2_set_learned_correction", "fa2_mlp_forward", "fa2_mlp_train_step",
    "fa2_learn_set_create", "fa2_learn_set_destroy", "fa2_learn_set_size", "fa2_learn_collect",
    "fa2_learn_set_read", "fa2_learn_fit", "fa2_mlp_launch_shape", "fa2_set_prevent_overlap",
)

FA2_OK = 0
FA2_NOALLOC_MAX_BODIES = 8192  # include/fa2b200.h
FA2_BATCH_MAX_NODES = 65536    # include/fa2b200.h
STATUS_NAMES = {
    0: "FA2_OK", 1: "FA2_ERR_INVALID_ARGUMENT", 2: "FA2_ERR_NO_DEVICE", 3: "FA2_ERR_CUDA",
    4: "FA2_ERR_OUT_OF_MEMORY", 5: "FA2_ERR_DEVICE_LIMIT", 6: "FA2_ERR_TOO_LARGE",
    7: "FA2_ERR_UNSUPPORTED", 8: "FA2_ERR_IO",
}


class GraphDesc(C.Structure):
    _fields_ = [("num_nodes", C.c_uint32), ("num_edges", C.c_uint64),
                ("sources", C.c_void_p), ("targets", C.c_void_p), ("weights", C.c_void_p)]


class Params(C.Structure):
    _fields_ = [("use_barneshut", C.c_int32), ("strong_gravity", C.c_int32),
                ("gravity", C.c_float), ("scale", C.c_float), ("theta", C.c_float),
                ("epssq", C.c_float), ("jitter_tolerance", C.c_float), ("k_s_max", C.c_float),
                ("device", C.c_int32), ("linlog", C.c_int32), ("multipole", C.c_int32),
                ("delta", C.c_float)]


class Stats(C.Structure):
    _fields_ = [("num_bodies", C.c_uint32), ("tree_nodes", C.c_uint32),
                ("tree_cells", C.c_uint32), ("max_level", C.c_int32),
                ("perturb_rounds", C.c_int32), ("device_error", C.c_int32),
                ("nnz_padded", C.c_uint64), ("global_speed", C.c_float),
                ("speed_efficiency", C.c_float), ("radius", C.c_float),
                ("root_x", C.c_float), ("root_y", C.c_float),
                ("interactions", C.c_uint64), ("visits", C.c_uint64),
                ("sort_passes", C.c_int32), ("learned_pairs", C.c_uint64)]


MLP_IN, MLP_HIDDEN, MLP_OUT = 12, 64, 2  # include/fa2b200.h


class Mlp(C.Structure):
    """fa2_mlp: the learned correction's FP32 parameters, [out][in] weights."""
    _fields_ = [("w1", C.c_float * (MLP_HIDDEN * MLP_IN)), ("b1", C.c_float * MLP_HIDDEN),
                ("w2", C.c_float * (MLP_HIDDEN * MLP_HIDDEN)), ("b2", C.c_float * MLP_HIDDEN),
                ("w3", C.c_float * (MLP_OUT * MLP_HIDDEN)), ("b3", C.c_float * MLP_OUT)]


class Fa2Error(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, str(status))
        text = _lib.fa2_status_string(status).decode() if _lib else name
        if _lib and status == 3:  # FA2_ERR_CUDA: the runtime's own error and where
            detail = _lib.fa2_last_cuda_error().decode()
            if detail:
                text = f"{text}: {detail}"
        super().__init__(f"{what}: {name} ({text})" if what else f"{name} ({text})")


_lib = None


def lib():
    """The loaded library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build the CUDA engine with `make -C {HERE}` "
            "(there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    vp, u32p, f32p = C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_float)
    ip = C.POINTER(C.c_int)
    L.fa2_default_params.argtypes = [C.POINTER(Params)]
    L.fa2_create.restype = vp
    L.fa2_create.argtypes = [C.POINTER(GraphDesc), C.POINTER(Params), ip]
    L.fa2_destroy.argtypes = [vp]
    L.fa2_set_positions.argtypes = [vp, vp]
    L.fa2_get_positions.argtypes = [vp, vp]
    L.fa2_step.argtypes = [vp, C.c_int32]
    L.fa2_step_timed.argtypes = [vp, C.c_int32, f32p, f32p, C.c_int32]
    L.fa2_step_host.argtypes = [vp, vp, C.c_int32, vp]
    L.fa2_kernel_name.restype = C.c_char_p
    L.fa2_kernel_name.argtypes = [C.c_int32]
    L.fa2_get_stats.argtypes = [vp, C.POINTER(Stats)]
    L.fa2_get_forces.argtypes = [vp, vp, vp]
    L.fa2_get_sort_order.argtypes = [vp, vp]
    L.fa2_set_speed_state.argtypes = [vp, C.c_float, C.c_float, vp]
    L.fa2_get_speed_state.argtypes = [vp, f32p, f32p, vp]
    L.fa2_set_force_params.argtypes = [vp, C.c_float, C.c_float]
    L.fa2_set_overlap.argtypes = [vp, C.c_int32]
    L.fa2_set_linlog.argtypes = [vp, C.c_int32]
    L.fa2_set_approximation.argtypes = [vp, C.c_float, C.c_int32]
    L.fa2_exact_repulsion.argtypes = [vp, C.c_int32, vp, vp]
    L.fa2_set_accuracy_guard.argtypes = [vp, C.c_int32, C.c_int32]
    L.fa2_get_accuracy_guard.argtypes = [vp, vp, vp, vp, vp]
    L.fa2_last_cuda_error.restype = C.c_char_p
    L.fa2_last_cuda_error.argtypes = []
    L.fa2_render_rgb.argtypes = [C.c_uint32, C.c_uint64, vp, vp, vp, C.c_int32, C.c_int32,
                                 C.c_int32, vp]
    L.fa2_png_encode.argtypes = [vp, C.c_int32, C.c_int32, C.c_char_p]
    L.fa2_write_png.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_char_p]
    L.fa2_batch_create.restype = vp
    L.fa2_batch_create.argtypes = [C.c_uint32, vp, C.POINTER(Params), ip]
    L.fa2_batch_destroy.argtypes = [vp]
    L.fa2_batch_set_positions.argtypes = [vp, vp]
    L.fa2_batch_get_positions.argtypes = [vp, vp]
    L.fa2_batch_step.argtypes = [vp, C.c_int32]
    L.fa2_batch_step_timed.argtypes = [vp, C.c_int32, f32p]
    L.fa2_batch_get_forces.argtypes = [vp, vp, vp]
    L.fa2_batch_get_sort_order.argtypes = [vp, vp]
    L.fa2_batch_configure.argtypes = [vp, C.c_uint32, C.c_int32, C.c_int32]
    L.fa2_batch_get_config.argtypes = [vp, vp, vp, vp]
    L.fa2_batch_autotune.argtypes = [vp, C.c_int32, vp, vp, vp, vp]
    L.fa2_batch_get_speed.argtypes = [vp, vp, vp]
    L.fa2_repulsion_noalloc.argtypes = [vp, vp, C.c_uint32, C.POINTER(Params), vp, vp]
    L.fa2_ugraph_load.restype = vp
    L.fa2_ugraph_load.argtypes = [C.c_char_p, ip]
    L.fa2_ugraph_from_pairs.restype = vp
    L.fa2_ugraph_from_pairs.argtypes = [vp, vp, C.c_uint64, ip]
    L.fa2_ugraph_free.argtypes = [vp]
    L.fa2_ugraph_num_nodes.restype = C.c_uint32
    L.fa2_ugraph_num_nodes.argtypes = [vp]
    L.fa2_ugraph_num_edges.restype = C.c_uint64
    L.fa2_ugraph_num_edges.argtypes = [vp]
    L.fa2_ugraph_node_map_r.argtypes = [vp, vp]
    L.fa2_ugraph_degrees.argtypes = [vp, vp]
    L.fa2_ugraph_edges.argtypes = [vp, vp, vp]
    L.fa2_random_positions.argtypes = [C.c_uint32, C.c_float, C.c_float, C.c_uint32, vp]
    L.fa2_write_layout.argtypes = [vp, vp, C.c_char_p, C.c_int]
    L.fa2_status_string.restype = C.c_char_p
    L.fa2_status_string.argtypes = [C.c_int]
    L.fa2_version.restype = C.c_char_p
    mp = C.POINTER(Mlp)
    L.fa2_mlp_init.argtypes = [mp, C.c_uint32]
    L.fa2_set_learned_correction.argtypes = [vp, mp]
    L.fa2_mlp_forward.argtypes = [C.c_int32, mp, vp, C.c_int64, vp]
    L.fa2_mlp_launch_shape.argtypes = [C.c_int32, vp, vp]
    L.fa2_set_prevent_overlap.argtypes = [vp, vp]
    L.fa2_mlp_train_step.argtypes = [C.c_int32, mp, mp, mp, C.c_int32, C.c_float, vp, vp, vp,
                                     C.c_int32, f32p]
    L.fa2_learn_set_create.restype = vp
    L.fa2_learn_set_create.argtypes = [C.c_int32, C.c_int64, ip]
    L.fa2_learn_set_destroy.argtypes = [vp]
    L.fa2_learn_set_size.restype = C.c_int64
    L.fa2_learn_set_size.argtypes = [vp]
    L.fa2_learn_collect.argtypes = [vp, vp, C.c_float, C.c_int32, C.POINTER(C.c_int64)]
    L.fa2_learn_set_read.argtypes = [vp, C.c_int64, C.c_int64, vp, vp, vp]
    L.fa2_learn_fit.argtypes = [vp, mp, C.c_int32, C.c_int32, C.c_float, C.c_uint32, f32p]
    _lib = L
    return L


def check(status: int, what: str = "") -> None:
    if status != FA2_OK:
        raise Fa2Error(status, what)

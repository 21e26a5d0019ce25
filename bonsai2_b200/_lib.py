"""ctypes binding of libbonsai_b200.so (the C ABI in include/bonsai_b200.h).

The library is the product: there is no Python or CPU fallback.  Loading
fails loudly if the in-tree shared library is missing.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# BONSAI_B200_LIB selects an alternative build of the same library (tuning
# builds, or the bounds-checked CHECKED_LIB_PATH)
LIB_PATH = os.environ.get("BONSAI_B200_LIB") or os.path.join(HERE, "libbonsai_b200.so")
CHECKED_LIB_PATH = os.path.join(HERE, "libbonsai_b200_checks.so")


class bonsai_params(ctypes.Structure):
    _fields_ = [("theta", ctypes.c_float), ("eps", ctypes.c_float), ("nleaf", ctypes.c_int),
                ("ncrit", ctypes.c_int), ("level_split", ctypes.c_int), ("dt", ctypes.c_float),
                ("device", ctypes.c_int)]


class bonsai_tree_info(ctypes.Structure):
    _fields_ = [("ncells", ctypes.c_int), ("nleaves", ctypes.c_int), ("nnodes", ctypes.c_int),
                ("nlevels", ctypes.c_int), ("ngroups", ctypes.c_int), ("status", ctypes.c_int),
                ("level_beg", ctypes.c_int * 32), ("level_end", ctypes.c_int * 32)]


# name -> (restype, argtypes); every entry point declared in include/bonsai_b200.h
P = ctypes.c_void_p
I = ctypes.c_int
SIGNATURES = {
    "bonsai_default_params": (None, [P]),
    "bonsai_create": (I, [P, P]),
    "bonsai_destroy": (I, [P]),
    "bonsai_alloc": (I, [P, I]),
    "bonsai_set_params": (I, [P, P]),
    "bonsai_set_particles": (I, [P, P, P, I]),
    "bonsai_set_particles_device": (I, [P, P, P, I]),
    "bonsai_get_particles": (I, [P, P, P, P]),
    "bonsai_get_particles_device": (I, [P, P, P, P]),
    "bonsai_set_particles_async": (I, [P, P, P, I]),
    "bonsai_get_particles_async": (I, [P, P, P, P]),
    "bonsai_build_tree": (I, [P, I]),
    "bonsai_compute_multipoles": (I, [P]),
    "bonsai_make_groups": (I, [P, I, I]),
    "bonsai_compute_forces": (I, [P, I, P]),
    "bonsai_move_particles": (I, [P]),
    "bonsai_compute_energies": (I, [P, P]),
    "bonsai_step": (I, [P, I, I]),
    "bonsai_step_timed": (I, [P, I, P]),
    "bonsai_graph_kernel_count": (I, [P]),
    "bonsai_get_stats": (I, [P, P]),
    "bonsai_fp32_peak": (I, [I, P]),
    "bonsai_binary_version": (I, [I, P, P]),
    "bonsai_selftest_wait_bound": (I, [I]),
    "bonsai_bounds_check": (I, [P, P, I]),
    "bonsai_bounds_selftest": (I, [I]),
    "bonsai_synchronize": (I, [P]),
    "bonsai_last_error": (I, [P]),
    "bonsai_step_graph": (I, [P, I]),
    "bonsai_stream": (P, [P]),
    "bonsai_copy_streams": (I, [P, P, P]),
    "bonsai_error_string": (ctypes.c_char_p, [I]),
    "bonsai_get_tree_info": (I, [P, P]),
    "bonsai_get_box": (I, [P, P]),
    "bonsai_get_keys": (I, [P, P, P, P, P, P]),
    "bonsai_get_cells": (I, [P, P, P, P, P, P, P, P]),
    "bonsai_get_groups": (I, [P, P]),
    "bonsai_get_walk_arrays": (I, [P, P, P, P, P]),
    "bonsai_direct_fp64": (I, [P, P, I, I, P]),
    "bonsai_direct_fp64_noalloc": (I, [P, I, P, I, ctypes.c_double, I, P, P]),
    "bonsai_set_theta_mode": (I, [P, I, ctypes.c_float, ctypes.c_float]),
    "bonsai_set_mlp_weights": (I, [P, P, I]),
    "bonsai_set_group_theta": (I, [P, P, I]),
    "bonsai_set_group_tau": (I, [P, P, I]),
    "bonsai_set_relative_bound": (I, [P, ctypes.c_float]),
    "bonsai_get_group_scale": (I, [P, P]),
    "bonsai_get_group_features": (I, [P, P, P]),
    "bonsai_get_group_theta": (I, [P, P]),
    "bonsai_get_group_interactions": (I, [P, P]),
    "bonsai_mlp_loss_grad": (I, [I, P, P, I, P, ctypes.c_float, ctypes.c_float, ctypes.c_float, P, P]),
    "bonsai_mlp_train": (I, [I, P, P, I, P, I, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, P]),
    "bonsai_mlp_predict": (I, [I, P, I, P, ctypes.c_float, ctypes.c_float, P]),
    "bonsai_set_precision": (I, [P, I]),
    "bonsai_set_particles_f64": (I, [P, P, P, I]),
    "bonsai_get_particles_f64": (I, [P, P, P, P]),
    "bonsai_set_systems": (I, [P, P, I]),
    "bonsai_get_system_energies": (I, [P, P]),
    "bonsai_set_walk_layout": (I, [P, I]),
    "bonsai_autotune": (I, [P, P, I, P, I, I, P, P]),
    "bonsai_plummer": (I, [ctypes.c_long, ctypes.c_uint, P, P]),
    "bonsai_galaxy": (I, [ctypes.c_long, ctypes.c_ulonglong, P, P]),
    "bonsai_read_tipsy": (I, [ctypes.c_char_p, P, P, P, P, P]),
    "bonsai_write_tipsy": (I, [ctypes.c_char_p, ctypes.c_double, I, I, P, P, P]),
    "bonsai_sync_velocities": (I, [P]),
    "bonsai_compute_forces_fp64": (I, [P, P, P]),
    "bonsai_set_block_steps": (I, [P, I, ctypes.c_float]),
    "bonsai_block_step": (I, [P, I]),
    "bonsai_get_levels": (I, [P, P]),
    "bonsai_clustered_field": (I, [ctypes.c_long, ctypes.c_ulonglong, I, P, P]),
    "bonsai_host_alloc": (P, [ctypes.c_size_t]),
    "bonsai_host_free": (None, [P]),
}

_lib = None


def load(path: str = LIB_PATH):
    """Load the in-tree CUDA library; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("libbonsai_b200.so not found at %s: run `python -m bonsai2_b200.build` "
                           "(there is no CPU fallback)" % path)
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


class BonsaiError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = load().bonsai_error_string(code)
        super().__init__("%s failed: %d (%s)" % (where, code, msg.decode() if msg else "?"))
        self.code = code

"""ctypes binding of libfluxion_b200.so (the C ABI in include/fluxion_b200.h).

The shared library is built in-tree next to this file. Importing this module
never falls back to anything else: a missing library raises at load time.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libfluxion_b200.so"

FX_OK = 0
FX_EINVAL = -1
FX_ENOMEM = -2
FX_ECUDA = -3
FX_ETIMEOUT = -4
FX_EADMIT = -5
FX_ENODEV = -6

FX_DCT_FP32 = 0
FX_DCT_TF32 = 1
FX_DCT_BF16 = 2
FX_DCT_SIMT = 3
FX_DCT_I8 = 4

FX_BH_FAST = 0
FX_BH_EXACT = 1

FX_LEAF_IEEE = 0
FX_LEAF_FAST = 1

STAGES = ["attract_integrate", "bh_keys", "bh_sort", "bh_tree", "bh_walk",
          "density", "congestion", "leaf", "fiedler", "attention"]

_CODES = {FX_EINVAL: "FX_EINVAL", FX_ENOMEM: "FX_ENOMEM", FX_ECUDA: "FX_ECUDA",
          FX_ETIMEOUT: "FX_ETIMEOUT", FX_EADMIT: "FX_EADMIT",
          FX_ENODEV: "FX_ENODEV"}


class FluxionError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code: int, where: str, message: str):
        super().__init__(f"{where}: {_CODES.get(code, code)}: {message}")
        self.code = code


class IterCfg(C.Structure):
    _fields_ = [("attract_weight", C.c_float), ("repel_weight", C.c_float),
                ("min_dist", C.c_float), ("theta", C.c_float),
                ("density_weight", C.c_float), ("target_density", C.c_float),
                ("density_bins", C.c_int32), ("dct_precision", C.c_int32),
                ("cong_cols", C.c_int32), ("cong_rows", C.c_int32),
                ("damping", C.c_float), ("dt", C.c_float), ("bh_walk", C.c_int32)]


class IterStats(C.Structure):
    _fields_ = [("hpwl", C.c_double), ("total_overflow", C.c_double),
                ("max_overflow", C.c_float), ("pad0", C.c_float),
                ("density_energy", C.c_double), ("iterations", C.c_int64),
                ("bh_nodes", C.c_int64)]


class LeafCfg(C.Structure):
    _fields_ = [("force_iterations", C.c_int32), ("attract_weight", C.c_float),
                ("repel_weight", C.c_float), ("damping", C.c_float),
                ("dt", C.c_float), ("schedule", C.c_int32),
                ("precision", C.c_int32), ("reserved1", C.c_int32)]


FX_LEAF_AUTO = 0
FX_LEAF_WARP = 1
FX_LEAF_CTA64 = 2
FX_LEAF_CTA128 = 3
FX_LEAF_CTA256 = 4
FX_LEAF_PER_CLUSTER = 5
FX_LEAF_PAIR64 = 6
FX_LEAF_PAIR128 = 7
FX_LEAF_PAIR256 = 8


class RefineCfg(C.Structure):
    _fields_ = [("max_iterations", C.c_int32), ("move_distance", C.c_float),
                ("overflow_threshold", C.c_float), ("grid_cols", C.c_int32),
                ("grid_rows", C.c_int32), ("reserved0", C.c_int32)]


class RefineStats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("moves", C.c_int64),
                ("total_overflow", C.c_float), ("max_overflow", C.c_float),
                ("hpwl", C.c_double)]


class PartCfg(C.Structure):
    _fields_ = [("max_leaf_size", C.c_int32), ("min_cluster_size", C.c_int32),
                ("balance_factor", C.c_float), ("power_iterations", C.c_int32),
                ("mode", C.c_int32), ("reserved0", C.c_int32), ("tol", C.c_double)]


class PartStats(C.Structure):
    _fields_ = [("n_leaves", C.c_int32), ("n_nodes", C.c_int32), ("max_depth", C.c_int32),
                ("levels", C.c_int32), ("power_iterations", C.c_int64)]


FX_PART_EXACT = 0
FX_PART_FP64 = 1

FX_JOB_PLACE = 0
FX_JOB_ECO = 1


class ServeCfg(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_int32), ("queue_capacity", C.c_int32),
                ("reserved0", C.c_int32), ("hbm_budget_bytes", C.c_int64)]


class JobDesc(C.Structure):
    _fields_ = [("kind", C.c_int32), ("keep_resident", C.c_int32), ("design_id", C.c_int64),
                ("n_gates", C.c_int32), ("n_nets", C.c_int32),
                ("net_ptr", C.c_void_p), ("net_gate", C.c_void_p),
                ("gate_w", C.c_void_p), ("gate_h", C.c_void_p),
                ("chip_w", C.c_float), ("chip_h", C.c_float),
                ("n_moves", C.c_int32), ("iterations", C.c_int32),
                ("move_gate", C.c_void_p), ("move_dx", C.c_void_p), ("move_dy", C.c_void_p),
                ("part", C.c_void_p), ("leaf", C.c_void_p), ("refine", C.c_void_p),
                ("iter", C.c_void_p)]


class JobResult(C.Structure):
    _fields_ = [("job_id", C.c_int64), ("design_id", C.c_int64), ("kind", C.c_int32),
                ("status", C.c_int32), ("n_gates", C.c_int32), ("n_leaves", C.c_int32),
                ("iterations", C.c_int32), ("max_overflow", C.c_float), ("hpwl", C.c_double),
                ("total_overflow", C.c_double), ("submit_s", C.c_double),
                ("start_s", C.c_double), ("end_s", C.c_double), ("est_bytes", C.c_int64),
                ("error", C.c_char * 160)]

P = C.c_void_p
I32 = C.c_int32
I64 = C.c_int64
F32 = C.c_float
PI32 = C.POINTER(C.c_int32)
PI64 = C.POINTER(C.c_int64)
PU32 = C.POINTER(C.c_uint32)
PF32 = C.POINTER(C.c_float)
PF64 = C.POINTER(C.c_double)

# name -> (restype, argtypes). Every symbol declared in include/fluxion_b200.h.
SIGNATURES = {
    "fx_last_error": (C.c_char_p, []),
    "fx_version": (C.c_char_p, []),
    "fx_ctx_create": (C.c_int, [C.POINTER(P), C.c_int]),
    "fx_ctx_destroy": (C.c_int, [P]),
    "fx_ctx_set_profiling": (C.c_int, [P, C.c_int]),
    "fx_ctx_set_profiling_stages": (C.c_int, [P, C.c_uint32]),
    "fx_ctx_stage_times": (C.c_int, [P, PF64, PI64, C.c_int]),
    "fx_ctx_reset_stage_times": (C.c_int, [P]),
    "fx_ctx_kernel_launches": (C.c_int64, [P]),
    "fx_ctx_mark": (C.c_int, [P, C.c_int]),
    "fx_ctx_elapsed": (C.c_int, [P, C.c_int, C.c_int, PF32]),
    "fx_ctx_synchronize": (C.c_int, [P]),
    "fx_design_load": (C.c_int, [P, I32, I32, PI32, PI32, PF32, PF32, F32, F32,
                                 C.POINTER(P)]),
    "fx_design_free": (C.c_int, [P]),
    "fx_design_sizes": (C.c_int, [P, PI64, PI64, PI64, PI64]),
    "fx_design_adjacency": (C.c_int, [P, PI32, PI32]),
    "fx_design_set_positions": (C.c_int, [P, PF32, PF32]),
    "fx_design_get_positions": (C.c_int, [P, PF32, PF32]),
    "fx_design_save_state": (C.c_int, [P]),
    "fx_design_trace": (C.c_int, [P, C.c_int]),
    "fx_design_leaf_trace_get": (C.c_int, [P, PF32, PF32]),
    "fx_stage_barnes_hut_walk": (C.c_int, [P, P, C.c_float, C.c_float, C.c_float, I32, PF32,
                                           PF32, C.POINTER(C.c_uint32), C.POINTER(C.c_int32),
                                           PF32, C.POINTER(C.c_int32)]),
    "fx_design_trace_get": (C.c_int, [P, PF32, PF32, PF32, PF32, PF32, PF32]),
    "fx_design_restore_state": (C.c_int, [P]),
    "fx_design_device_bytes": (C.c_int64, [P]),
    "fx_congestion": (C.c_int, [P, P, PF32, PF32, I32, I32, PU32, PF64, PF64, PF32]),
    # device pointers throughout
    "fx_congestion_noalloc": (C.c_int, [P, P, P, P, I32, I32, P, P, P]),
    "fx_iter_cfg_default": (C.c_int, [C.POINTER(IterCfg)]),
    "fx_force_iterate": (C.c_int, [P, P, C.POINTER(IterCfg), I32, PF32, PF32,
                                   C.POINTER(IterStats)]),
    "fx_stage_attraction": (C.c_int, [P, P, F32, PF32, PF32]),
    "fx_stage_barnes_hut": (C.c_int, [P, P, F32, F32, F32, PF32, PF32, PU32,
                                      PI32, PF32]),
    "fx_stage_density": (C.c_int, [P, P, I32, F32, F32, I32, PF32, PF32, PF32,
                                   PF32, PF32, PF32, PF64]),
    "fx_adjacency_build": (C.c_int64, [I32, I32, PI32, PI32, PI32, PI32, C.c_int64]),
    "fx_leaf_cfg_default": (C.c_int, [C.POINTER(LeafCfg)]),
    "fx_hapr_place_leaves": (C.c_int, [P, P, I32, PI32, PI32, PF32, C.POINTER(LeafCfg),
                                       PF32, PF32, PI32]),
    "fx_fiedler": (C.c_int, [P, P, I32, PI32, PI32, I32, C.c_double, PF32, PI32, PF64]),
    "fx_refine_cfg_default": (C.c_int, [C.POINTER(RefineCfg)]),
    "fx_part_cfg_default": (C.c_int, [C.POINTER(PartCfg)]),
    "fx_attention": (C.c_int, [P, P, I32, PI32, PI32, I32, PI32, PF32]),
    "fx_attention_tree": (C.c_int, [P, P, I32, PI32, PI32, PI32, I32, I32, PI32, PI32, PI32,
                                    C.c_int64, PI32]),
    "fx_blif_read": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, I32]),
    "fx_def_write": (C.c_int, [C.c_char_p, C.c_char_p, I32, PF32, PF32, F32, F32, C.c_char_p]),
    "fx_serve_cfg_default": (C.c_int, [C.POINTER(ServeCfg)]),
    "fx_serve_estimate": (C.c_int, [C.POINTER(JobDesc), PI64]),
    "fx_serve_create": (C.c_int, [C.POINTER(ServeCfg), C.POINTER(C.c_void_p)]),
    "fx_serve_destroy": (C.c_int, [P]),
    "fx_serve_submit": (C.c_int, [P, C.POINTER(JobDesc), PI64]),
    "fx_serve_poll": (C.c_int, [P, I32, C.POINTER(JobResult)]),
    "fx_serve_positions": (C.c_int, [P, I64, PF32, PF32]),
    "fx_serve_release": (C.c_int, [P, I64]),
    "fx_serve_stats": (C.c_int, [P, PI64, PI32, PI32, PI32, PI64]),
    "fx_partition": (C.c_int, [P, P, C.POINTER(PartCfg), I32, PI32, PI32, PF32, PI32,
                               C.POINTER(PartStats)]),
    "fx_refine": (C.c_int, [P, P, C.POINTER(RefineCfg), PF32, PF32, C.POINTER(RefineStats),
                            PU32]),
    "fx_synth_plain": (C.c_int, [C.c_uint64, I32, I32, F32, F32, I32, C.POINTER(P)]),
    "fx_synth_leaves": (C.c_int, [C.c_uint64, I32, I32, I32, F32, C.POINTER(P)]),
    "fx_netlist_sizes": (C.c_int, [P, PI64, PI64, PI64, PI64]),
    "fx_netlist_copy": (C.c_int, [P, PI32, PI32, PF32, PF32, PF32, PF32, PF32,
                                  PI32, PF32]),
    "fx_netlist_free": (C.c_int, [P]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the in-tree library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FluxionError(FX_ENODEV, "load",
                           f"{LIB_PATH} is missing; build it with "
                           "`python -c 'import __graft_entry__ as g; g.build()'`")
    lib = C.CDLL(str(LIB_PATH), mode=os.RTLD_NOW | os.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, where: str) -> int:
    if rc < 0:
        msg = load().fx_last_error()
        raise FluxionError(rc, where, msg.decode() if msg else "")
    return rc


def ptr(a, ctype):
    """Pointer to a contiguous numpy array (or NULL for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))

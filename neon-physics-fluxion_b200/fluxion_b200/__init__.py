"""fluxion_b200 -- B200-native HAPR placement hot path (FLUXION v4 drop-in).

Compute runs in libfluxion_b200.so (hand-written sm_100a CUDA behind the C ABI
of include/fluxion_b200.h); this package is the host-side mirror of the
reference's data types and entry points.
"""
from ._lib import (FX_BH_EXACT, FX_BH_FAST, FX_LEAF_FAST, FX_LEAF_IEEE, FX_DCT_BF16, FX_DCT_FP32, FX_DCT_I8, FX_DCT_SIMT, FX_DCT_TF32, FX_LEAF_AUTO,
                   FX_LEAF_CTA64, FX_LEAF_CTA128, FX_LEAF_CTA256, FX_LEAF_PAIR64,
                   FX_LEAF_PAIR128, FX_LEAF_PAIR256, FX_LEAF_PER_CLUSTER,
                   FX_LEAF_WARP, FX_PART_EXACT, FX_PART_FP64, FluxionError, IterCfg,
                   IterStats, LeafCfg, PartCfg, load)
from .api import (Circuit, Context, Design, Placement, RoutingGrid, Server, Synth,
                  build_adjacency, build_and_compute, compute_congestion, compute_hpwl, default_context,
                  hierarchy_levels, iter_cfg, top_k_lists, leaf_cfg, part_cfg, read_blif, refine_cfg, serve_estimate,
                  synth_leaves, synth_plain, write_def)
from . import engine
from .engine import FluxionEngine

__all__ = [
    "Circuit", "Context", "Design", "Placement", "RoutingGrid", "Synth",
    "build_adjacency", "build_and_compute", "compute_congestion", "compute_hpwl", "default_context",
    "iter_cfg", "synth_leaves", "synth_plain", "FluxionError", "IterCfg", "IterStats",
    "load", "FX_BH_FAST", "FX_BH_EXACT", "FX_LEAF_IEEE", "FX_LEAF_FAST", "FX_DCT_FP32", "FX_DCT_TF32", "FX_DCT_BF16", "FX_DCT_SIMT", "FX_DCT_I8", "leaf_cfg",
    "LeafCfg", "FX_LEAF_AUTO", "FX_LEAF_WARP", "FX_LEAF_CTA64", "FX_LEAF_CTA128",
    "FX_LEAF_CTA256", "FX_LEAF_PAIR64", "FX_LEAF_PAIR128", "FX_LEAF_PAIR256",
    "FX_LEAF_PER_CLUSTER", "refine_cfg", "part_cfg", "PartCfg",
    "FX_PART_EXACT", "FX_PART_FP64", "Server", "serve_estimate", "read_blif", "write_def",
    "FluxionEngine", "hierarchy_levels", "top_k_lists",
]

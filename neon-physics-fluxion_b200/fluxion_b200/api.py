"""Host-side mirror of the reference's data types and entry points.

The reference (HAPR_fluxion_v4, Rust) keeps a Circuit of flat per-gate arrays
(src/data/circuit.rs:43-78), a Placement of per-gate f32 positions
(src/data/placement.rs:9-24) and a RoutingGrid (src/data/grid.rs:10-21).
The same shapes are kept here as numpy arrays, and every compute entry point
runs on the B200 through the C ABI in include/fluxion_b200.h. There is no CPU
compute path in this package.
"""
from __future__ import annotations

import atexit
import ctypes as C
import weakref
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import FluxionError, IterCfg, IterStats, check, load, ptr


# ---------------------------------------------------------------------------
# data types
@dataclass
class Circuit:
    """Flat netlist: net e joins net_gate[net_ptr[e]:net_ptr[e+1]].

    Mirrors Circuit (circuit.rs:43-78): gate_widths/gate_heights per gate,
    net_gate_indices per net (here as CSR), chip_width/chip_height.
    """
    num_gates: int
    net_ptr: np.ndarray
    net_gate: np.ndarray
    gate_widths: np.ndarray
    gate_heights: np.ndarray
    chip_width: float
    chip_height: float
    name: str = "design"
    gate_names: Optional[list] = None

    @property
    def num_nets(self) -> int:
        return int(self.net_ptr.shape[0] - 1)

    @property
    def num_pins(self) -> int:
        return int(self.net_ptr[-1])

    @property
    def net_gate_indices(self) -> list:
        p, g = self.net_ptr, self.net_gate
        return [g[p[e]:p[e + 1]].tolist() for e in range(self.num_nets)]

    @staticmethod
    def from_nets(nets: Sequence[Sequence[int]], num_gates: int,
                  chip_width: float = 1000.0, chip_height: float = 1000.0,
                  gate_widths=None, gate_heights=None, name: str = "design",
                  gate_names=None) -> "Circuit":
        ptr_ = np.zeros(len(nets) + 1, np.int32)
        for e, n in enumerate(nets):
            ptr_[e + 1] = ptr_[e] + len(n)
        flat = np.fromiter((g for n in nets for g in n), np.int32, int(ptr_[-1]))
        w = np.full(num_gates, 2.0, np.float32) if gate_widths is None else \
            np.asarray(gate_widths, np.float32)
        h = np.full(num_gates, 10.0, np.float32) if gate_heights is None else \
            np.asarray(gate_heights, np.float32)
        return Circuit(num_gates, ptr_, flat, w, h, float(chip_width),
                       float(chip_height), name, gate_names)


@dataclass
class Placement:
    """Per-gate f32 positions and quality metrics (placement.rs:9-24)."""
    gate_x: np.ndarray
    gate_y: np.ndarray
    total_wirelength: float = 0.0
    max_congestion: float = 0.0
    wns: float = 0.0
    runtime_ms: float = 0.0

    @staticmethod
    def new(num_gates: int) -> "Placement":
        return Placement(np.zeros(num_gates, np.float32), np.zeros(num_gates, np.float32))

    def set_position(self, g: int, x: float, y: float) -> None:
        self.gate_x[g] = x
        self.gate_y[g] = y


@dataclass
class RoutingGrid:
    """Routing grid geometry and congestion (grid.rs:10-32).

    h_congestion and v_congestion are f32 arrays of rows*cols (row-major),
    equal to each other as in the reference; counts holds the exact uint32
    crossing counts they were converted from.
    """
    cols: int
    rows: int
    cell_width: float
    cell_height: float
    h_congestion: np.ndarray
    v_congestion: np.ndarray
    capacity: np.ndarray
    counts: Optional[np.ndarray] = None

    @staticmethod
    def new(chip_width: float, chip_height: float, cols: int, rows: int) -> "RoutingGrid":
        cw = np.float32(chip_width) / np.float32(cols)
        ch = np.float32(chip_height) / np.float32(rows)
        cap = (cw + ch) * np.float32(0.5)
        cells = cols * rows
        return RoutingGrid(cols, rows, float(cw), float(ch),
                           np.zeros(cells, np.float32), np.zeros(cells, np.float32),
                           np.full(cells, cap, np.float32))

    def cell_index(self, col: int, row: int) -> int:
        return row * self.cols + col

    def cell_at(self, x: float, y: float):
        """grid.rs:58-62: f32 division, saturating cast, clamp to the grid."""
        def one(v, cell, n):
            q = np.float32(v) / np.float32(cell)
            if not (q >= 1.0):
                return 0
            return int(min(int(q) if q < 2.0 ** 63 else n - 1, n - 1))
        return one(x, self.cell_width, self.cols), one(y, self.cell_height, self.rows)

    def cell_center(self, col: int, row: int):
        return ((np.float32(col) + np.float32(0.5)) * np.float32(self.cell_width),
                (np.float32(row) + np.float32(0.5)) * np.float32(self.cell_height))

    def overflow(self) -> np.ndarray:
        return np.maximum((self.h_congestion + self.v_congestion) - self.capacity,
                          np.float32(0.0))

    def max_overflow(self) -> float:
        return float(self.overflow().max(initial=0.0))

    def total_overflow(self) -> float:
        return float(self.overflow().astype(np.float64).sum())


# ---------------------------------------------------------------------------
# Handles still open when the interpreter exits are closed by an exit hook,
# designs and servers before the contexts they run on, while every object and
# the CUDA runtime are still alive (the teardown of module globals frees them
# in no particular order).
_OPEN = {"design": weakref.WeakSet(), "server": weakref.WeakSet(), "ctx": weakref.WeakSet()}


@atexit.register
def _close_open_handles() -> None:
    for kind in ("design", "server", "ctx"):
        for obj in list(_OPEN[kind]):
            try:
                obj.close()
            except Exception:
                pass


# ---------------------------------------------------------------------------
# device context and resident designs
class Context:
    """A CUDA context on one B200 (fx_ctx)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = C.c_void_p()
        check(self.lib.fx_ctx_create(C.byref(h), device), "fx_ctx_create")
        self.handle = h
        _OPEN["ctx"].add(self)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.fx_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_profiling(self, on: bool = True, stages=None) -> None:
        """Per-stage event timing on or off; `stages` (names from STAGES)
        limits it to those stages, None times all of them."""
        mask = 0xFFFFFFFF if stages is None else sum(1 << _lib.STAGES.index(s) for s in stages)
        check(self.lib.fx_ctx_set_profiling_stages(self.handle, mask), "set_profiling_stages")
        check(self.lib.fx_ctx_set_profiling(self.handle, int(on)), "set_profiling")

    def stage_times(self) -> dict:
        n = len(_lib.STAGES)
        ms = (C.c_double * n)()
        calls = (C.c_int64 * n)()
        check(self.lib.fx_ctx_stage_times(self.handle, ms, calls, n), "stage_times")
        return {s: (ms[i], calls[i]) for i, s in enumerate(_lib.STAGES)}

    def reset_stage_times(self) -> None:
        check(self.lib.fx_ctx_reset_stage_times(self.handle), "reset_stage_times")

    def kernel_launches(self) -> int:
        return int(self.lib.fx_ctx_kernel_launches(self.handle))

    def mark(self, slot: int) -> None:
        check(self.lib.fx_ctx_mark(self.handle, slot), "fx_ctx_mark")

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float()
        check(self.lib.fx_ctx_elapsed(self.handle, a, b, C.byref(ms)), "fx_ctx_elapsed")
        return ms.value

    def synchronize(self) -> None:
        check(self.lib.fx_ctx_synchronize(self.handle), "fx_ctx_synchronize")


class Design:
    """A device-resident netlist (fx_design) with positions and workspaces."""

    def __init__(self, ctx: Context, circuit: Circuit):
        self.ctx = ctx
        self.lib = ctx.lib
        self.circuit = circuit
        net_ptr = np.ascontiguousarray(circuit.net_ptr, np.int32)
        net_gate = np.ascontiguousarray(circuit.net_gate, np.int32)
        w = np.ascontiguousarray(circuit.gate_widths, np.float32)
        h = np.ascontiguousarray(circuit.gate_heights, np.float32)
        d = C.c_void_p()
        check(self.lib.fx_design_load(ctx.handle, circuit.num_gates, circuit.num_nets,
                                      ptr(net_ptr, C.c_int32), ptr(net_gate, C.c_int32),
                                      ptr(w, C.c_float), ptr(h, C.c_float),
                                      circuit.chip_width, circuit.chip_height,
                                      C.byref(d)), "fx_design_load")
        self.handle = d
        _OPEN["design"].add(self)
        n, m, p, a = (C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64())
        check(self.lib.fx_design_sizes(d, C.byref(n), C.byref(m), C.byref(p),
                                       C.byref(a)), "fx_design_sizes")
        self.n, self.m, self.p, self.a = n.value, m.value, p.value, a.value

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.fx_design_free(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def adjacency(self):
        ap = np.zeros(self.n + 1, np.int32)
        ai = np.zeros(max(self.a, 1), np.int32)
        check(self.lib.fx_design_adjacency(self.handle, ptr(ap, C.c_int32),
                                           ptr(ai, C.c_int32)), "fx_design_adjacency")
        return ap, ai[:self.a]

    def set_positions(self, x, y) -> None:
        x = np.ascontiguousarray(x, np.float32)
        y = np.ascontiguousarray(y, np.float32)
        check(self.lib.fx_design_set_positions(self.handle, ptr(x, C.c_float),
                                               ptr(y, C.c_float)), "set_positions")

    def get_positions(self):
        x = np.empty(self.n, np.float32)
        y = np.empty(self.n, np.float32)
        check(self.lib.fx_design_get_positions(self.handle, ptr(x, C.c_float),
                                               ptr(y, C.c_float)), "get_positions")
        return x, y

    def save_state(self) -> None:
        """Device-side checkpoint of positions and velocities."""
        check(self.lib.fx_design_save_state(self.handle), "save_state")

    def restore_state(self) -> None:
        """Restores the last save_state (stream-ordered, no host sync)."""
        check(self.lib.fx_design_restore_state(self.handle), "restore_state")

    def trace(self, enable: bool = True) -> None:
        """fx_design_trace: record each plain iteration's total force and start state."""
        check(self.lib.fx_design_trace(self.handle, 1 if enable else 0), "fx_design_trace")

    def trace_get(self) -> dict:
        """The last traced iteration: total force fx, fy and the positions x0, y0 and
        velocities vx0, vy0 it started from (float32 arrays of n)."""
        out = {k: np.empty(self.n, np.float32) for k in ("fx", "fy", "x0", "y0", "vx0", "vy0")}
        check(self.lib.fx_design_trace_get(self.handle, *[ptr(out[k], C.c_float) for k in
                                                          ("fx", "fy", "x0", "y0", "vx0", "vy0")]),
              "fx_design_trace_get")
        return out

    def leaf_trace_get(self, slots: int):
        """fx_design_leaf_trace_get: each slot's first-iteration force (fx, fy) of the
        last traced leaf batch, in leaf_gate order."""
        fx = np.empty(slots, np.float32)
        fy = np.empty(slots, np.float32)
        check(self.lib.fx_design_leaf_trace_get(self.handle, ptr(fx, C.c_float),
                                                ptr(fy, C.c_float)), "fx_design_leaf_trace_get")
        return fx, fy

    def device_bytes(self) -> int:
        return int(self.lib.fx_design_device_bytes(self.handle))

    # -- rows D+F -----------------------------------------------------------
    def congestion(self, cols: int, rows: int, x=None, y=None):
        """Returns (counts[rows*cols] uint32, hpwl f64, total_overflow, max_overflow)."""
        counts = np.empty(cols * rows, np.uint32)
        hp, tot, mx = C.c_double(), C.c_double(), C.c_float()
        xa = None if x is None else np.ascontiguousarray(x, np.float32)
        ya = None if y is None else np.ascontiguousarray(y, np.float32)
        check(self.lib.fx_congestion(self.ctx.handle, self.handle, ptr(xa, C.c_float),
                                     ptr(ya, C.c_float), cols, rows,
                                     ptr(counts, C.c_uint32), C.byref(hp),
                                     C.byref(tot), C.byref(mx)), "fx_congestion")
        return counts, hp.value, tot.value, mx.value

    # -- single stages --------------------------------------------------------
    def attraction(self, k: float = 1.0):
        fx = np.empty(self.n, np.float32)
        fy = np.empty(self.n, np.float32)
        check(self.lib.fx_stage_attraction(self.ctx.handle, self.handle, k,
                                           ptr(fx, C.c_float), ptr(fy, C.c_float)),
              "fx_stage_attraction")
        return fx, fy

    def barnes_hut(self, k: float = 0.5, theta: float = 0.5, min_dist: float = 0.1,
                   walk: int = _lib.FX_BH_EXACT, terms: bool = False):
        """fx_stage_barnes_hut_walk: forces, keys (gate order), sorted order and root
        square; with terms=True (FX_BH_FAST only) also each gate's interaction count."""
        fx = np.empty(self.n, np.float32)
        fy = np.empty(self.n, np.float32)
        keys = np.empty(self.n, np.uint32)
        perm = np.empty(self.n, np.int32)
        root = np.empty(3, np.float32)
        cnt = np.empty(self.n, np.int32) if terms else None
        check(self.lib.fx_stage_barnes_hut_walk(self.ctx.handle, self.handle, k, theta,
                                                min_dist, walk, ptr(fx, C.c_float),
                                                ptr(fy, C.c_float), ptr(keys, C.c_uint32),
                                                ptr(perm, C.c_int32), ptr(root, C.c_float),
                                                ptr(cnt, C.c_int32)),
              "fx_stage_barnes_hut_walk")
        if terms:
            return fx, fy, keys, perm, root, cnt
        return fx, fy, keys, perm, root

    def density(self, bins: int, target: float = 0.7, weight: float = 1.0,
                precision: int = _lib.FX_DCT_SIMT, grids: bool = False):
        fx = np.empty(self.n, np.float32)
        fy = np.empty(self.n, np.float32)
        g = [np.empty(bins * bins, np.float32) for _ in range(4)] if grids else [None] * 4
        e = C.c_double()
        check(self.lib.fx_stage_density(self.ctx.handle, self.handle, bins, target, weight,
                                        precision, ptr(fx, C.c_float), ptr(fy, C.c_float),
                                        *(ptr(a, C.c_float) for a in g), C.byref(e)),
              "fx_stage_density")
        out = {"fx": fx, "fy": fy, "energy": e.value}
        if grids:
            out.update(rho=g[0].reshape(bins, bins), phi=g[1].reshape(bins, bins),
                       ex=g[2].reshape(bins, bins), ey=g[3].reshape(bins, bins))
        return out

    # -- row H: batched leaf placement ------------------------------------------
    def place_leaves(self, leaf_ptr, leaf_gate, region, cfg=None, x=None, y=None):
        """placer.rs:65-69 + place_gates_in_leaf for every leaf in one launch.

        Returns (x, y, schedule): positions of all gates (leaf gates placed,
        others taken from x/y or zero) and the schedule the call used."""
        cfg = cfg if cfg is not None else leaf_cfg()
        lp = np.ascontiguousarray(leaf_ptr, np.int32)
        lg = np.ascontiguousarray(leaf_gate, np.int32)
        rg = np.ascontiguousarray(region, np.float32).reshape(-1)
        ox = np.zeros(self.n, np.float32) if x is None else np.array(x, np.float32)
        oy = np.zeros(self.n, np.float32) if y is None else np.array(y, np.float32)
        sched = C.c_int32()
        check(self.lib.fx_hapr_place_leaves(self.ctx.handle, self.handle, len(lp) - 1,
                                            ptr(lp, C.c_int32), ptr(lg, C.c_int32),
                                            ptr(rg, C.c_float), C.byref(cfg),
                                            ptr(ox, C.c_float), ptr(oy, C.c_float),
                                            C.byref(sched)), "fx_hapr_place_leaves")
        return ox, oy, sched.value

    # -- row G: batched power iteration -----------------------------------------
    def fiedler(self, cluster_ptr, cluster_gate, max_iters: int = 30, tol: float = 0.0):
        """partitioner.rs:106-185 for every cluster at once.

        Returns (v[G] f32 in cluster_gate order, iterations[C], lambda[C])."""
        cp = np.ascontiguousarray(cluster_ptr, np.int32)
        cg = np.ascontiguousarray(cluster_gate, np.int32)
        C_ = len(cp) - 1
        v = np.empty(len(cg), np.float32)
        its = np.empty(C_, np.int32)
        lam = np.empty(C_, np.float64)
        check(self.lib.fx_fiedler(self.ctx.handle, self.handle, C_, ptr(cp, C.c_int32),
                                  ptr(cg, C.c_int32), max_iters, tol, ptr(v, C.c_float),
                                  ptr(its, C.c_int32), ptr(lam, C.c_double)), "fx_fiedler")
        return v, its, lam

    def congestion_noalloc(self, cols: int, rows: int, d_counts: int, d_x: int = 0,
                           d_y: int = 0, d_hpwl_overflow: int = 0,
                           d_max_overflow: int = 0) -> None:
        """fx_congestion_noalloc: device pointers (ints, 0 = NULL) in and out,
        enqueued on the context's stream without allocating; synchronize the
        context before reading the outputs."""
        vp = lambda a: C.c_void_p(a) if a else None
        check(self.lib.fx_congestion_noalloc(self.ctx.handle, self.handle, vp(d_x), vp(d_y),
                                             cols, rows, vp(d_counts), vp(d_hpwl_overflow),
                                             vp(d_max_overflow)), "fx_congestion_noalloc")

    # -- hierarchy build ---------------------------------------------------------
    def partition(self, cfg=None) -> dict:
        """build_hierarchy (partitioner.rs:36-100) + leaf regions (placer.rs:40-63):
        leaf_ptr[L+1], leaf_gate[N], region[L, 4] = (cx, cy, w, h), leaf_depth[L],
        and the fx_part_stats fields."""
        cfg = cfg if cfg is not None else part_cfg()
        cap = self.n + 1
        lp = np.zeros(cap + 1, np.int32)
        lg = np.zeros(max(self.n, 1), np.int32)
        rg = np.zeros(4 * cap, np.float32)
        ld = np.zeros(cap, np.int32)
        st = _lib.PartStats()
        check(self.lib.fx_partition(self.ctx.handle, self.handle, C.byref(cfg), cap,
                                    ptr(lp, C.c_int32), ptr(lg, C.c_int32),
                                    ptr(rg, C.c_float), ptr(ld, C.c_int32), C.byref(st)),
              "fx_partition")
        L = st.n_leaves
        return dict(leaf_ptr=lp[:L + 1], leaf_gate=lg[:self.n], region=rg[:4 * L].reshape(L, 4),
                    leaf_depth=ld[:L], num_nodes=st.n_nodes, max_depth=st.max_depth,
                    levels=st.levels, power_iterations=st.power_iterations)

    # -- (f.4) attention scores between the clusters of one level ----------------
    def attention_level(self, cluster_ptr, cluster_gate, top_k: int = 10,
                        scores: bool = False):
        """compute_level_attention (attention.rs:50-88) for one level's clusters
        (CSR over gates). Returns (top[n, top_k] int32, -1 padded; scores[n, n]
        f32 or None)."""
        cp = np.ascontiguousarray(cluster_ptr, np.int32)
        cg = np.ascontiguousarray(cluster_gate, np.int32)
        n = len(cp) - 1
        top = np.full((n, top_k), -1, np.int32)
        sc = np.zeros((n, n), np.float32) if scores else None
        check(self.lib.fx_attention(self.ctx.handle, self.handle, n, ptr(cp, C.c_int32),
                                    ptr(cg, C.c_int32), top_k, ptr(top, C.c_int32),
                                    ptr(sc, C.c_float)), "fx_attention")
        return top, sc

    def attention(self, tree: dict, top_k: int = 10, scores: bool = False) -> list:
        """compute_all_attention (attention.rs:33-48) over a hierarchy from
        partition(): one dict(level_index, top_k, scores) per depth with at
        least two clusters. top_k is an (n, top_k) int32 array, each row the
        AttentionLevel.top_k list padded with -1 (top_k_lists() gives the
        lists). Without scores the whole hierarchy goes to fx_attention_tree
        in one call; with them each level is an fx_attention call (dense
        n x n)."""
        if not scores:
            lp = np.ascontiguousarray(tree["leaf_ptr"], np.int32)
            lg = np.ascontiguousarray(tree["leaf_gate"], np.int32)
            ld = np.ascontiguousarray(tree["leaf_depth"], np.int32)
            L = len(lp) - 1
            cap = 64
            depth = np.zeros(cap, np.int32)
            count = np.zeros(cap, np.int32)
            top = np.full(max(1, 2 * L * top_k), -1, np.int32)
            nl = C.c_int32()
            check(self.lib.fx_attention_tree(self.ctx.handle, self.handle, L,
                                             ptr(lp, C.c_int32), ptr(lg, C.c_int32),
                                             ptr(ld, C.c_int32), top_k, cap, C.byref(nl),
                                             ptr(depth, C.c_int32), ptr(count, C.c_int32),
                                             len(top), ptr(top, C.c_int32)),
                  "fx_attention_tree")
            out, off = [], 0
            for v in range(nl.value):
                n = int(count[v])
                rows = top[off:off + n * top_k].reshape(n, top_k) if top_k else \
                    np.zeros((n, 0), np.int32)
                out.append(dict(level_index=int(depth[v]), top_k=rows, scores=None))
                off += n * top_k
            return out
        out = []
        for depth, (cp, cg) in enumerate(hierarchy_levels(tree["leaf_ptr"], tree["leaf_gate"],
                                                          tree["leaf_depth"])):
            if len(cp) - 1 < 2:
                continue
            top, sc = self.attention_level(cp, cg, top_k, scores)
            out.append(dict(level_index=depth, top_k=top, scores=sc))
        return out

    # -- congestion refinement ----------------------------------------------------
    def refine(self, cfg=None, x=None, y=None, counts: bool = False):
        """refiner.rs:34-126 refine_placement. With x/y (host arrays, updated
        in place) or on the resident positions. Returns RefineStats (and the
        final counts when counts=True)."""
        cfg = cfg if cfg is not None else refine_cfg()
        st = _lib.RefineStats()
        xa = None if x is None else np.ascontiguousarray(x, np.float32)
        ya = None if y is None else np.ascontiguousarray(y, np.float32)
        cnt = np.empty(cfg.grid_cols * cfg.grid_rows, np.uint32) if counts else None
        check(self.lib.fx_refine(self.ctx.handle, self.handle, C.byref(cfg),
                                 ptr(xa, C.c_float), ptr(ya, C.c_float), C.byref(st),
                                 ptr(cnt, C.c_uint32)), "fx_refine")
        if x is not None:
            x[...] = xa
            y[...] = ya
        return (st, cnt) if counts else st

    # -- the plain composite iteration -------------------------------------
    def force_iterate(self, cfg: "IterCfg", iters: int, x=None, y=None) -> IterStats:
        st = IterStats()
        xa = None if x is None else np.ascontiguousarray(x, np.float32)
        ya = None if y is None else np.ascontiguousarray(y, np.float32)
        check(self.lib.fx_force_iterate(self.ctx.handle, self.handle, C.byref(cfg), iters,
                                        ptr(xa, C.c_float), ptr(ya, C.c_float),
                                        C.byref(st)), "fx_force_iterate")
        if x is not None and xa is not x:
            x[...] = xa
        if y is not None and ya is not y:
            y[...] = ya
        return st


def top_k_lists(top) -> list:
    """AttentionLevel.top_k (attention.rs:15) from a -1 padded top-k array."""
    return [[int(j) for j in r if j >= 0] for r in np.asarray(top)]


def hierarchy_levels(leaf_ptr, leaf_gate, leaf_depth) -> list:
    """HierarchyTree::clusters_at_depth (hierarchy.rs:134-159) for every depth
    0..max_depth of a hierarchy given by its leaves in DFS order and their
    depths (recursive_bisect makes two children per internal node,
    partitioner.rs:85-99, so the depths fix the tree): a list over depth of
    (cluster_ptr, cluster_gate), the clusters in DFS order, each cluster's
    gates those of its leaves in order."""
    lp = np.asarray(leaf_ptr, np.int64)
    lg = np.asarray(leaf_gate, np.int32)
    d = [int(v) for v in leaf_depth]
    L = len(d)
    if L == 0:
        return []
    # path of each leaf as a binary code of d[i] bits (0 = first child)
    code = [0] * L
    for i in range(1, L):
        c = code[i - 1] + 1
        if d[i] >= d[i - 1]:
            c <<= d[i] - d[i - 1]
        else:
            k = d[i - 1] - d[i]
            if c & ((1 << k) - 1):
                raise ValueError("leaf depths do not form a full binary tree")
            c >>= k
        code[i] = c
    if code[-1] + 1 != 1 << d[-1] or code[0] != 0:
        raise ValueError("leaf depths do not form a full binary tree")
    wide = max(d) > 62
    dd = np.asarray(d, np.int64)
    cc = np.asarray(code, object if wide else np.int64)
    size = np.diff(lp)
    levels = []
    for t in range(max(d) + 1):
        idx = np.nonzero(dd >= t)[0]
        pre = cc[idx] >> (dd[idx] - t).astype(cc.dtype)
        first = np.ones(len(idx), bool)
        first[1:] = pre[1:] != pre[:-1]
        run = np.cumsum(first) - 1
        csize = np.bincount(run, weights=size[idx], minlength=int(first.sum())).astype(np.int64)
        cp = np.zeros(len(csize) + 1, np.int32)
        cp[1:] = np.cumsum(csize)
        cg = np.concatenate([lg[lp[i]:lp[i + 1]] for i in idx]) if len(idx) else lg[:0]
        levels.append((cp, cg.astype(np.int32)))
    return levels


def leaf_cfg(**overrides) -> "_lib.LeafCfg":
    cfg = _lib.LeafCfg()
    check(load().fx_leaf_cfg_default(C.byref(cfg)), "fx_leaf_cfg_default")
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


# ---------------------------------------------------------------------------
# serving
def _addr(a) -> Optional[int]:
    return None if a is None else a.ctypes.data


class Server:
    """fx_server: placement (PLACE) and ECO jobs admitted by device footprint
    and run `slots` at a time, each on its own worker context."""

    def __init__(self, device: int = 0, slots: int = 8, hbm_budget_bytes: int = 0,
                 queue_capacity: int = 65536):
        self.lib = load()
        cfg = _lib.ServeCfg()
        check(self.lib.fx_serve_cfg_default(C.byref(cfg)), "fx_serve_cfg_default")
        cfg.device, cfg.slots = device, slots
        cfg.hbm_budget_bytes, cfg.queue_capacity = hbm_budget_bytes, queue_capacity
        h = C.c_void_p()
        check(self.lib.fx_serve_create(C.byref(cfg), C.byref(h)), "fx_serve_create")
        self.handle = h
        _OPEN["server"].add(self)

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.fx_serve_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def place_desc(circuit: Circuit, keep_resident: bool = False, part=None, leaf=None,
                   refine=None):
        """(JobDesc, arrays it points to) for a PLACE job."""
        arrs = [np.ascontiguousarray(circuit.net_ptr, np.int32),
                np.ascontiguousarray(circuit.net_gate, np.int32),
                np.ascontiguousarray(circuit.gate_widths, np.float32),
                np.ascontiguousarray(circuit.gate_heights, np.float32)]
        cfgs = [part, leaf, refine]
        d = _lib.JobDesc(kind=_lib.FX_JOB_PLACE, keep_resident=int(keep_resident),
                         n_gates=circuit.num_gates, n_nets=circuit.num_nets,
                         net_ptr=_addr(arrs[0]), net_gate=_addr(arrs[1]),
                         gate_w=_addr(arrs[2]), gate_h=_addr(arrs[3]),
                         chip_w=circuit.chip_width, chip_h=circuit.chip_height,
                         part=C.addressof(part) if part is not None else None,
                         leaf=C.addressof(leaf) if leaf is not None else None,
                         refine=C.addressof(refine) if refine is not None else None)
        return d, (arrs, cfgs)

    @staticmethod
    def eco_desc(design_id: int, gates, dx, dy, iterations: int = 50, iter_cfg=None,
                 n_gates: int = 0):
        arrs = [np.ascontiguousarray(gates, np.int32), np.ascontiguousarray(dx, np.float32),
                np.ascontiguousarray(dy, np.float32)]
        d = _lib.JobDesc(kind=_lib.FX_JOB_ECO, design_id=design_id, n_gates=n_gates,
                         n_moves=len(arrs[0]), iterations=iterations,
                         move_gate=_addr(arrs[0]), move_dx=_addr(arrs[1]),
                         move_dy=_addr(arrs[2]),
                         iter=C.addressof(iter_cfg) if iter_cfg is not None else None)
        return d, (arrs, [iter_cfg])

    def submit(self, desc_and_keep) -> int:
        desc, _keep = desc_and_keep
        jid = C.c_int64()
        check(self.lib.fx_serve_submit(self.handle, C.byref(desc), C.byref(jid)),
              "fx_serve_submit")
        return jid.value

    def submit_place(self, circuit: Circuit, keep_resident: bool = False, **cfgs) -> int:
        return self.submit(self.place_desc(circuit, keep_resident, **cfgs))

    def submit_eco(self, design_id: int, gates, dx, dy, iterations: int = 50,
                   iter_cfg=None) -> int:
        return self.submit(self.eco_desc(design_id, gates, dx, dy, iterations, iter_cfg))

    def poll(self, wait_ms: int = -1) -> Optional[dict]:
        r = _lib.JobResult()
        got = self.lib.fx_serve_poll(self.handle, wait_ms, C.byref(r))
        if got < 0:
            check(got, "fx_serve_poll")
        if got == 0:
            return None
        out = {k: getattr(r, k) for k, _ in _lib.JobResult._fields_ if k != "error"}
        out["error"] = r.error.decode(errors="replace")
        return out

    def positions(self, design_id: int, n: int):
        x = np.empty(n, np.float32)
        y = np.empty(n, np.float32)
        check(self.lib.fx_serve_positions(self.handle, design_id, ptr(x, C.c_float),
                                          ptr(y, C.c_float)), "fx_serve_positions")
        return x, y

    def release(self, design_id: int) -> None:
        check(self.lib.fx_serve_release(self.handle, design_id), "fx_serve_release")

    def stats(self) -> dict:
        rb, q, r, res, ln = C.c_int64(), C.c_int32(), C.c_int32(), C.c_int32(), C.c_int64()
        check(self.lib.fx_serve_stats(self.handle, C.byref(rb), C.byref(q), C.byref(r),
                                      C.byref(res), C.byref(ln)), "fx_serve_stats")
        return dict(reserved_bytes=rb.value, queued=q.value, running=r.value,
                    resident=res.value, launches=ln.value)


def serve_estimate(desc_and_keep) -> int:
    """Host-only admission estimate (bytes) of a job description."""
    desc, _ = desc_and_keep
    out = C.c_int64()
    check(load().fx_serve_estimate(C.byref(desc), C.byref(out)), "fx_serve_estimate")
    return out.value


def part_cfg(**overrides) -> "_lib.PartCfg":
    cfg = _lib.PartCfg()
    check(load().fx_part_cfg_default(C.byref(cfg)), "fx_part_cfg_default")
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


def refine_cfg(**overrides) -> "_lib.RefineCfg":
    cfg = _lib.RefineCfg()
    check(load().fx_refine_cfg_default(C.byref(cfg)), "fx_refine_cfg_default")
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


def iter_cfg(**overrides) -> IterCfg:
    cfg = IterCfg()
    check(load().fx_iter_cfg_default(C.byref(cfg)), "fx_iter_cfg_default")
    for k, v in overrides.items():
        if not hasattr(cfg, k):
            raise KeyError(k)
        setattr(cfg, k, v)
    return cfg


# ---------------------------------------------------------------------------
# reference entry points
_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def compute_congestion(grid: RoutingGrid, placement: Placement, circuit: Circuit,
                       design: Optional[Design] = None) -> RoutingGrid:
    """congestion.rs:11-62 compute_congestion_cpu, on the GPU.

    Fills grid.h_congestion / grid.v_congestion (identical f32 grids) and
    grid.counts from the exact device counts.
    """
    own = design is None
    if own:
        design = Design(default_context(), circuit)
    try:
        counts, hpwl, _, _ = design.congestion(grid.cols, grid.rows,
                                               placement.gate_x, placement.gate_y)
    finally:
        if own:
            design.close()
    grid.counts = counts
    grid.h_congestion = counts.astype(np.float32)
    grid.v_congestion = grid.h_congestion.copy()
    return grid


def build_and_compute(placement: Placement, circuit: Circuit, cols: int, rows: int,
                      design: Optional[Design] = None) -> RoutingGrid:
    """congestion.rs:65-74 build_and_compute."""
    grid = RoutingGrid.new(circuit.chip_width, circuit.chip_height, cols, rows)
    return compute_congestion(grid, placement, circuit, design)


def compute_hpwl(placement: Placement, circuit: Circuit,
                 design: Optional[Design] = None) -> float:
    """placement.rs:48-74 compute_hpwl, summed in FP64 on the GPU."""
    own = design is None
    if own:
        design = Design(default_context(), circuit)
    try:
        _, hpwl, _, _ = design.congestion(1, 1, placement.gate_x, placement.gate_y)
    finally:
        if own:
            design.close()
    return hpwl


def build_adjacency(circuit: Circuit):
    """circuit.rs:154-171 Circuit::build_adjacency, in the reference's order.

    Host-only (no GPU); returns (adj_ptr[N+1], adj_idx[A]) int32 CSR."""
    lib = load()
    net_ptr = np.ascontiguousarray(circuit.net_ptr, np.int32)
    net_gate = np.ascontiguousarray(circuit.net_gate, np.int32)
    ap = np.zeros(circuit.num_gates + 1, np.int32)
    a = check(lib.fx_adjacency_build(circuit.num_gates, circuit.num_nets,
                                     ptr(net_ptr, C.c_int32), ptr(net_gate, C.c_int32),
                                     ptr(ap, C.c_int32), None, 0), "fx_adjacency_build")
    ai = np.zeros(max(a, 1), np.int32)
    check(lib.fx_adjacency_build(circuit.num_gates, circuit.num_nets,
                                 ptr(net_ptr, C.c_int32), ptr(net_gate, C.c_int32),
                                 ptr(ap, C.c_int32), ptr(ai, C.c_int32), a),
          "fx_adjacency_build")
    return ap, ai[:a]


# ---------------------------------------------------------------------------
# synthetic netlists (host-only, no GPU needed)
@dataclass
class Synth:
    circuit: Circuit
    placement: Placement
    leaf_ptr: np.ndarray
    region: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))


def _netlist_out(h) -> Synth:
    lib = load()
    n, m, p, nl = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
    check(lib.fx_netlist_sizes(h, C.byref(n), C.byref(m), C.byref(p), C.byref(nl)),
          "fx_netlist_sizes")
    N, M, Pn, L = n.value, m.value, p.value, nl.value
    net_ptr = np.empty(M + 1, np.int32)
    net_gate = np.empty(max(Pn, 1), np.int32)
    w = np.empty(N, np.float32)
    hh = np.empty(N, np.float32)
    x = np.empty(N, np.float32)
    y = np.empty(N, np.float32)
    die = np.empty(2, np.float32)
    leaf_ptr = np.empty(L + 1, np.int32)
    region = np.empty(4 * max(L, 1), np.float32)
    check(lib.fx_netlist_copy(h, ptr(net_ptr, C.c_int32), ptr(net_gate, C.c_int32),
                              ptr(w, C.c_float), ptr(hh, C.c_float), ptr(x, C.c_float),
                              ptr(y, C.c_float), ptr(die, C.c_float),
                              ptr(leaf_ptr, C.c_int32), ptr(region, C.c_float)),
          "fx_netlist_copy")
    lib.fx_netlist_free(h)
    circ = Circuit(N, net_ptr, net_gate[:Pn], w, hh, float(die[0]), float(die[1]),
                   name="synthetic")
    return Synth(circ, Placement(x, y), leaf_ptr, region[:4 * L])


def read_blif(path) -> Circuit:
    """parser::blif::parse (H/src/parser/blif.rs:12-116) -> Circuit (gates g0..,
    width 2, height 10, die 1000 x 1000, named after the file stem)."""
    h = C.c_void_p()
    name = C.create_string_buffer(256)
    check(load().fx_blif_read(str(path).encode(), C.byref(h), name, 256), "fx_blif_read")
    s = _netlist_out(h)
    c = s.circuit
    c.name = name.value.decode()
    c.gate_names = [f"g{i}" for i in range(c.num_gates)]
    return c


def write_def(path, circuit: Circuit, placement: Placement) -> None:
    """parser::def::write_def (H/src/parser/def.rs:11-43)."""
    names = None
    if circuit.gate_names is not None:
        names = b"".join(n.encode() + b"\0" for n in circuit.gate_names)
    x = np.ascontiguousarray(placement.gate_x, np.float32)
    y = np.ascontiguousarray(placement.gate_y, np.float32)
    check(load().fx_def_write(str(path).encode(), circuit.name.encode(), circuit.num_gates,
                              ptr(x, C.c_float), ptr(y, C.c_float), circuit.chip_width,
                              circuit.chip_height, names), "fx_def_write")


def synth_plain(seed: int, n_gates: int, n_nets: int, die: float,
                leaf_size: int = 64) -> Synth:
    """Seeded plain netlist (see fx_synth_plain in include/fluxion_b200.h)."""
    h = C.c_void_p()
    check(load().fx_synth_plain(seed, n_gates, n_nets, die, die, leaf_size, C.byref(h)),
          "fx_synth_plain")
    return _netlist_out(h)


def synth_leaves(seed: int, n_clusters: int, min_size: int = 16, max_size: int = 128,
                 nets_per_gate: float = 1.5) -> Synth:
    """Seeded batch of independent leaf clusters (fx_synth_leaves)."""
    h = C.c_void_p()
    check(load().fx_synth_leaves(seed, n_clusters, min_size, max_size, nets_per_gate,
                                 C.byref(h)), "fx_synth_leaves")
    return _netlist_out(h)

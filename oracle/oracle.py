"""CPU oracle for the HAPR placement hot path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
this module; the product never does.

* liboracle.so  -- C++ restatement of the reference's Rust CPU path
  (HAPR_fluxion_v4/src/...; see fx_oracle.cpp for the per-function citations)
  plus the Barnes-Hut tree rules of neon_old_codebase/src/cpp/BarnesHutTree.cpp
  restated on the Morton radix tree with FP64 accumulation.
* _ref/libbh_ref.so -- the reference's own BarnesHutTree.cpp compiled from the
  reference sources (Makefile target `ref`), when it was built.
* DCT Poisson density in FP64: a restatement of ElectrostaticSmoothingForce
  (neon_old_codebase/src/python/fluxion/force_electrostatic.py:47-150) on the
  reference's own third-party dependency, scipy.fft (dctn/idctn, type 2,
  norm='ortho'; scipy 1.18.1 in this image, unpinned by the reference).
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "_build" / "liboracle.so"
REF_LIB = HERE / "_ref" / "libbh_ref.so"

_lib = None
_ref = None

I32P = C.POINTER(C.c_int32)
I64P = C.POINTER(C.c_int64)
U32P = C.POINTER(C.c_uint32)
F32P = C.POINTER(C.c_float)
F64P = C.POINTER(C.c_double)


def build() -> None:
    """Builds the oracle libraries (output goes to stderr, never stdout)."""
    import sys
    r = subprocess.run(["make", "-s", "-C", str(HERE)], stdout=subprocess.PIPE,
                       stderr=subprocess.STDOUT, text=True)
    if r.stdout:
        sys.stderr.write(r.stdout)
    r.check_returncode()


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        L = C.CDLL(str(LIB))
        L.or_cell_at.restype = C.c_int64
        L.or_cell_at.argtypes = [C.c_float, C.c_float, C.c_int64]
        L.or_grid_geometry.argtypes = [C.c_float, C.c_float, C.c_int64, C.c_int64,
                                       F32P, F32P, F32P]
        L.or_congestion.argtypes = [C.c_int32, I32P, I32P, F32P, F32P, C.c_float,
                                    C.c_float, C.c_int64, C.c_int64, F32P, F32P]
        L.or_congestion_parallel.argtypes = [C.c_int32, I32P, I32P, F32P, F32P, C.c_float,
                                             C.c_float, C.c_int64, C.c_int64, C.c_int32,
                                             F32P, F32P]
        L.or_congestion_sample.argtypes = [C.c_int32, I32P, I32P, F32P, F32P, C.c_float,
                                           C.c_float, C.c_int64, C.c_int64, C.c_int32,
                                           F32P, F32P]
        L.or_refine.restype = C.c_int32
        L.or_refine.argtypes = [C.c_int32, C.c_int32, I32P, I32P, F32P, F32P, C.c_float,
                                C.c_float, C.c_int32, C.c_float, C.c_float, C.c_int64,
                                C.c_int64, F32P]
        L.or_overflow.argtypes = [F32P, F32P, C.c_int64, C.c_int64, C.c_float, F32P, F32P]
        L.or_hpwl_f32.restype = C.c_float
        L.or_hpwl_f32.argtypes = [C.c_int32, I32P, I32P, F32P, F32P]
        L.or_hpwl_f64.restype = C.c_double
        L.or_hpwl_f64.argtypes = [C.c_int32, I32P, I32P, F32P, F32P]
        L.or_build_adjacency.restype = C.c_int64
        L.or_build_adjacency.argtypes = [C.c_int32, C.c_int32, I32P, I32P, I32P, I32P,
                                         C.c_int64]
        L.or_attraction_f32.argtypes = [C.c_int32, I32P, I32P, F32P, F32P, C.c_float,
                                        F32P, F32P]
        L.or_attraction_f64.argtypes = [C.c_int32, I32P, I32P, F32P, F32P, C.c_double,
                                        F64P, F64P]
        L.or_integrate.argtypes = [C.c_int32, F32P, F32P, F32P, F32P, F32P, F32P,
                                   C.c_float, C.c_float, C.c_float, C.c_float,
                                   C.c_float, C.c_float]
        L.or_place_leaf.argtypes = [C.c_int32, I32P, I32P, I32P, C.c_float, C.c_float,
                                    C.c_float, C.c_float, C.c_int32, C.c_float,
                                    C.c_float, C.c_float, C.c_float, F32P, F32P]
        L.or_leaf_forces_f64.argtypes = [C.c_int32, I32P, I32P, I32P, F32P, F32P,
                                         C.c_double, C.c_double, F64P, F64P]
        L.or_build_hierarchy.restype = C.c_int32
        L.or_build_hierarchy.argtypes = [C.c_int32, I32P, I32P, C.c_int32, C.c_int32,
                                         C.c_float, C.c_int32, C.c_float, C.c_float,
                                         I32P, I32P, F32P, I32P, I32P, I32P]
        L.or_fiedler_vector.argtypes = [I32P, I32P, C.c_int32, I32P, C.c_int32, F32P]
        L.or_bh_root.argtypes = [C.c_int32, F32P, F32P, F32P]
        L.or_bh_keys.argtypes = [C.c_int32, F32P, F32P, F32P, U32P]
        L.or_bh_forces.argtypes = [C.c_int32, F32P, F32P, C.c_double, C.c_float,
                                   C.c_double, F64P, F64P, U32P, I32P, F32P, I64P,
                                   C.c_int32, F32P, F32P]
        L.or_repulsion_exact.argtypes = [C.c_int32, F32P, F32P, C.c_double, C.c_double,
                                         F64P, F64P]
        L.or_attention_sample.argtypes = [C.c_int32, I32P, I32P, C.c_int32, I32P, I32P,
                                          C.c_int32, I32P, C.c_int32, F32P, I32P, F64P]
        L.or_congestion_counts.argtypes = [C.c_int32, I32P, I32P, F32P, F32P, C.c_float,
                                           C.c_float, C.c_int64, C.c_int64, U32P]
        _lib = L
    return _lib


def ref_lib():
    """The reference's own BarnesHutTree.cpp, or None when it was not built."""
    global _ref
    if _ref is None and REF_LIB.exists():
        R = C.CDLL(str(REF_LIB))
        R.bh_ref_forces.argtypes = [C.c_int, F64P, F64P, F64P, C.c_double, C.c_double,
                                    C.c_double, F64P, F64P, C.c_int]
        R.bh_ref_forces_sample.argtypes = [C.c_int, F64P, F64P, F64P, C.c_double,
                                           C.c_double, C.c_double, F64P, F64P, C.c_int,
                                           C.c_int]
        _ref = R
    return _ref


_synth = None


def synth_lib() -> C.CDLL:
    """oracle/_build/libsynth.so: the seeded workload generator without the
    CUDA library (for the CPU reference arm)."""
    global _synth
    if _synth is None:
        L = C.CDLL(str(HERE / "_build" / "libsynth.so"))
        L.fx_synth_plain.argtypes = [C.c_uint64, C.c_int32, C.c_int32, C.c_float, C.c_float,
                                     C.c_int32, C.POINTER(C.c_void_p)]
        L.fx_netlist_sizes.argtypes = [C.c_void_p] + [C.POINTER(C.c_int64)] * 4
        L.fx_netlist_copy.argtypes = [C.c_void_p] + [C.c_void_p] * 9
        L.fx_netlist_free.argtypes = [C.c_void_p]
        L.or_synth_last_error.restype = C.c_char_p
        _synth = L
    return _synth


def synth_plain(seed, n_gates, n_nets, die, leaf_size=64):
    """The plain workload generator (fx_synth_plain) through libsynth.so:
    a namespace with the netlist CSR (net_ptr, net_gate), gate_widths,
    gate_heights, chip_width, chip_height, num_gates and the seeded start
    positions gate_x, gate_y -- the same bytes the GPU arm generates."""
    from types import SimpleNamespace
    L = synth_lib()
    h = C.c_void_p()
    if L.fx_synth_plain(seed, n_gates, n_nets, die, die, leaf_size, C.byref(h)) != 0:
        raise RuntimeError(L.or_synth_last_error().decode())
    n, m, p, nl = (C.c_int64() for _ in range(4))
    L.fx_netlist_sizes(h, C.byref(n), C.byref(m), C.byref(p), C.byref(nl))
    N, M, P = n.value, m.value, p.value
    a = dict(net_ptr=np.empty(M + 1, np.int32), net_gate=np.empty(max(P, 1), np.int32),
             gate_widths=np.empty(N, np.float32), gate_heights=np.empty(N, np.float32),
             gate_x=np.empty(N, np.float32), gate_y=np.empty(N, np.float32))
    dd = np.empty(2, np.float32)
    lp = np.empty(nl.value + 1, np.int32)
    rg = np.empty(4 * max(nl.value, 1), np.float32)
    L.fx_netlist_copy(h, *(a[k].ctypes.data for k in ("net_ptr", "net_gate", "gate_widths",
                                                      "gate_heights", "gate_x", "gate_y")),
                      dd.ctypes.data, lp.ctypes.data, rg.ctypes.data)
    L.fx_netlist_free(h)
    a["net_gate"] = a["net_gate"][:P]
    return SimpleNamespace(num_gates=N, num_nets=M, num_pins=P, chip_width=float(dd[0]),
                           chip_height=float(dd[1]), **a)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


# ---- grid / congestion / HPWL (grid.rs, congestion.rs, placement.rs) -------
def cell_at(v: float, cell: float, n: int) -> int:
    return int(lib().or_cell_at(v, cell, n))


def grid_geometry(chip_w, chip_h, cols, rows):
    cw, ch, cap = C.c_float(), C.c_float(), C.c_float()
    lib().or_grid_geometry(chip_w, chip_h, cols, rows, C.byref(cw), C.byref(ch),
                           C.byref(cap))
    return cw.value, ch.value, cap.value


def congestion(net_ptr, net_gate, x, y, chip_w, chip_h, cols, rows):
    net_ptr, net_gate, x, y = _i32(net_ptr), _i32(net_gate), _f32(x), _f32(y)
    h = np.empty(cols * rows, np.float32)
    v = np.empty(cols * rows, np.float32)
    lib().or_congestion(len(net_ptr) - 1, _p(net_ptr, C.c_int32), _p(net_gate, C.c_int32),
                        _p(x, C.c_float), _p(y, C.c_float), chip_w, chip_h, cols, rows,
                        _p(h, C.c_float), _p(v, C.c_float))
    return h, v


def congestion_parallel(net_ptr, net_gate, x, y, chip_w, chip_h, cols, rows, threads):
    """compute_congestion_cpu's literal loops (congestion.rs:11-62) over all
    nets on `threads` host threads (per-thread grids summed in order; the
    counts are exact integers, so h and v equal the single-threaded loop's)."""
    h = np.empty(rows * cols, np.float32)
    v = np.empty(rows * cols, np.float32)
    lib().or_congestion_parallel(len(net_ptr) - 1, _p(_i32(net_ptr), C.c_int32),
                                 _p(_i32(net_gate), C.c_int32), _p(_f32(x), C.c_float),
                                 _p(_f32(y), C.c_float), chip_w, chip_h, cols, rows, threads,
                                 _p(h, C.c_float), _p(v, C.c_float))
    return h, v


def congestion_counts(net_ptr, net_gate, x, y, chip_w, chip_h, cols, rows):
    """The counts of compute_congestion_cpu (h == v) through a difference array:
    O(nets + cells), for full-size netlists."""
    net_ptr, net_gate, x, y = _i32(net_ptr), _i32(net_gate), _f32(x), _f32(y)
    out = np.empty(cols * rows, np.uint32)
    lib().or_congestion_counts(len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                               _p(net_gate, C.c_int32), _p(x, C.c_float), _p(y, C.c_float),
                               chip_w, chip_h, cols, rows, _p(out, C.c_uint32))
    return out


def congestion_sample(net_ptr, net_gate, x, y, chip_w, chip_h, cols, rows, stride):
    net_ptr, net_gate, x, y = _i32(net_ptr), _i32(net_gate), _f32(x), _f32(y)
    h = np.empty(cols * rows, np.float32)
    v = np.empty(cols * rows, np.float32)
    lib().or_congestion_sample(len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                               _p(net_gate, C.c_int32), _p(x, C.c_float), _p(y, C.c_float),
                               chip_w, chip_h, cols, rows, stride, _p(h, C.c_float),
                               _p(v, C.c_float))
    return h, v


def refine(net_ptr, net_gate, x, y, chip_w, chip_h, max_iters=100, move_distance=5.0,
           threshold=1.0, cols=256, rows=256):
    """refiner.rs:34-126 on float32 copies of x/y; returns (x, y, iters, stats)."""
    net_ptr, net_gate = _i32(net_ptr), _i32(net_gate)
    x, y = np.array(x, np.float32), np.array(y, np.float32)
    out = np.zeros(3, np.float32)
    it = lib().or_refine(len(x), len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                         _p(net_gate, C.c_int32), _p(x, C.c_float), _p(y, C.c_float),
                         chip_w, chip_h, max_iters, move_distance, threshold, cols, rows,
                         _p(out, C.c_float))
    return x, y, int(it), dict(total_overflow=float(out[0]), max_overflow=float(out[1]),
                               hpwl_f32=float(out[2]))


def overflow(h, v, cols, rows, capacity):
    t, m = C.c_float(), C.c_float()
    lib().or_overflow(_p(_f32(h), C.c_float), _p(_f32(v), C.c_float), cols, rows,
                      capacity, C.byref(t), C.byref(m))
    return t.value, m.value


def hpwl_f32(net_ptr, net_gate, x, y) -> float:
    net_ptr, net_gate, x, y = _i32(net_ptr), _i32(net_gate), _f32(x), _f32(y)
    return float(lib().or_hpwl_f32(len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                                   _p(net_gate, C.c_int32), _p(x, C.c_float),
                                   _p(y, C.c_float)))


def hpwl_f64(net_ptr, net_gate, x, y) -> float:
    net_ptr, net_gate, x, y = _i32(net_ptr), _i32(net_gate), _f32(x), _f32(y)
    return float(lib().or_hpwl_f64(len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                                   _p(net_gate, C.c_int32), _p(x, C.c_float),
                                   _p(y, C.c_float)))


# ---- adjacency / attraction / integrate (circuit.rs, placer.rs) ------------
def build_adjacency(n, net_ptr, net_gate):
    net_ptr, net_gate = _i32(net_ptr), _i32(net_gate)
    ap = np.zeros(n + 1, np.int32)
    cap = 0
    total = lib().or_build_adjacency(n, len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                                     _p(net_gate, C.c_int32), _p(ap, C.c_int32),
                                     None, cap)
    ai = np.zeros(max(total, 1), np.int32)
    lib().or_build_adjacency(n, len(net_ptr) - 1, _p(net_ptr, C.c_int32),
                             _p(net_gate, C.c_int32), _p(ap, C.c_int32),
                             _p(ai, C.c_int32), total)
    return ap, ai[:total]


def attraction_f32(adj_ptr, adj_idx, x, y, k=1.0):
    n = len(adj_ptr) - 1
    fx, fy = np.empty(n, np.float32), np.empty(n, np.float32)
    lib().or_attraction_f32(n, _p(_i32(adj_ptr), C.c_int32), _p(_i32(adj_idx), C.c_int32),
                            _p(_f32(x), C.c_float), _p(_f32(y), C.c_float), k,
                            _p(fx, C.c_float), _p(fy, C.c_float))
    return fx, fy


def attraction_f64(adj_ptr, adj_idx, x, y, k=1.0):
    n = len(adj_ptr) - 1
    fx, fy = np.empty(n), np.empty(n)
    adj_ptr, adj_idx, x, y = _i32(adj_ptr), _i32(adj_idx), _f32(x), _f32(y)
    lib().or_attraction_f64(n, _p(adj_ptr, C.c_int32), _p(adj_idx, C.c_int32),
                            _p(x, C.c_float), _p(y, C.c_float), k,
                            _p(fx, C.c_double), _p(fy, C.c_double))
    return fx, fy


def integrate(x, y, vx, vy, fx, fy, dt, damping, box):
    """In place on float32 arrays (placer.rs:275-280)."""
    n = len(x)
    lib().or_integrate(n, _p(x, C.c_float), _p(y, C.c_float), _p(vx, C.c_float),
                       _p(vy, C.c_float), _p(_f32(fx), C.c_float),
                       _p(_f32(fy), C.c_float), dt, damping, *box)


def place_leaf(gates, adj_ptr, adj_idx, region, iters, attract=1.0, repel=0.5,
               damping=0.9, dt=0.1, out_x=None, out_y=None, n_total=None):
    gates = _i32(gates)
    if out_x is None:
        n_total = n_total if n_total is not None else int(gates.max()) + 1
        out_x = np.zeros(n_total, np.float32)
        out_y = np.zeros(n_total, np.float32)
    if len(gates) == 0:
        return out_x, out_y
    adj_ptr, adj_idx = _i32(adj_ptr), _i32(adj_idx)
    lib().or_place_leaf(len(gates), _p(gates, C.c_int32), _p(adj_ptr, C.c_int32),
                        _p(adj_idx, C.c_int32), *[float(r) for r in region], iters,
                        attract, repel, damping, dt, _p(out_x, C.c_float),
                        _p(out_y, C.c_float))
    return out_x, out_y


def leaf_forces_f64(gates, adj_ptr, adj_idx, px, py, attract=1.0, repel=0.5):
    gates = _i32(gates)
    n = len(gates)
    fx, fy = np.empty(n), np.empty(n)
    adj_ptr, adj_idx, px, py = _i32(adj_ptr), _i32(adj_idx), _f32(px), _f32(py)
    lib().or_leaf_forces_f64(n, _p(gates, C.c_int32), _p(adj_ptr, C.c_int32),
                             _p(adj_idx, C.c_int32), _p(px, C.c_float), _p(py, C.c_float),
                             attract, repel, _p(fx, C.c_double), _p(fy, C.c_double))
    return fx, fy


# ---- hierarchy (partitioner.rs, placer.rs region pass) ---------------------
def build_hierarchy(n, adj_ptr, adj_idx, chip_w, chip_h, max_leaf=64, min_cluster=8,
                    balance=0.4, iters=30):
    adj_ptr, adj_idx = _i32(adj_ptr), _i32(adj_idx)
    cap_l = max(2 * n // max(1, min(max_leaf, min_cluster) // 2) + 2, 4)
    lp = np.zeros(cap_l + 1, np.int32)
    lg = np.zeros(n, np.int32)
    rg = np.zeros(4 * cap_l, np.float32)
    ld = np.zeros(cap_l, np.int32)
    nodes, md = C.c_int32(), C.c_int32()
    L = lib().or_build_hierarchy(n, _p(adj_ptr, C.c_int32), _p(adj_idx, C.c_int32),
                                 max_leaf, min_cluster, balance, iters, chip_w, chip_h,
                                 _p(lp, C.c_int32), _p(lg, C.c_int32), _p(rg, C.c_float),
                                 _p(ld, C.c_int32), C.byref(nodes), C.byref(md))
    return dict(leaf_ptr=lp[:L + 1], leaf_gate=lg, region=rg[:4 * L].reshape(L, 4),
                leaf_depth=ld[:L], num_nodes=nodes.value, max_depth=md.value)


def fiedler_vector(adj_ptr, adj_idx, gates, iters=30):
    gates = _i32(gates)
    out = np.empty(len(gates), np.float32)
    lib().or_fiedler_vector(_p(_i32(adj_ptr), C.c_int32), _p(_i32(adj_idx), C.c_int32),
                            len(gates), _p(gates, C.c_int32), iters, _p(out, C.c_float))
    return out


# ---- Barnes-Hut ------------------------------------------------------------
def bh_root(x, y):
    x, y = _f32(x), _f32(y)
    r = np.empty(3, np.float32)
    lib().or_bh_root(len(x), _p(x, C.c_float), _p(y, C.c_float), _p(r, C.c_float))
    return r


def bh_keys(x, y, root):
    x, y, root = _f32(x), _f32(y), _f32(root)
    k = np.empty(len(x), np.uint32)
    lib().or_bh_keys(len(x), _p(x, C.c_float), _p(y, C.c_float), _p(root, C.c_float),
                     _p(k, C.c_uint32))
    return k


def bh_forces(x, y, k=0.5, theta=0.5, min_dist=0.1, threads=1):
    """Barnes-Hut forces with the device's tree and opening decisions.

    Returns the FP64 recomputation of each point's interaction list (fx, fy)
    and the f32 forces in the device's operation order (fx32, fy32). min_dist
    enters the FP64 law as given; the decisions and the f32 law use its f32
    rounding. Pass float(np.float32(v)) to compare with a device run.
    """
    x, y = _f32(x), _f32(y)
    n = len(x)
    fx, fy = np.empty(n), np.empty(n)
    fx32, fy32 = np.empty(n, np.float32), np.empty(n, np.float32)
    keys = np.empty(n, np.uint32)
    perm = np.empty(n, np.int32)
    root = np.empty(3, np.float32)
    inter = np.empty(n, np.int64)
    lib().or_bh_forces(n, _p(x, C.c_float), _p(y, C.c_float), k, theta, min_dist,
                       _p(fx, C.c_double), _p(fy, C.c_double), _p(keys, C.c_uint32),
                       _p(perm, C.c_int32), _p(root, C.c_float), _p(inter, C.c_int64),
                       threads, _p(fx32, C.c_float), _p(fy32, C.c_float))
    return dict(fx=fx, fy=fy, fx32=fx32, fy32=fy32, keys=keys, perm=perm, root=root,
                interactions=inter)


def repulsion_exact(x, y, k=0.5, min_dist=0.1):
    x, y = _f32(x), _f32(y)
    n = len(x)
    fx, fy = np.empty(n), np.empty(n)
    lib().or_repulsion_exact(n, _p(x, C.c_float), _p(y, C.c_float), k, min_dist,
                             _p(fx, C.c_double), _p(fy, C.c_double))
    return fx, fy


def bh_reference(x, y, k=0.5, theta=0.5, min_dist=0.1, threads=1, stride=1):
    """Forces from the reference's own BarnesHutTree.cpp (unit charges).

    stride > 1 evaluates only every stride-th point (a timing sample; the
    other entries are left as zero)."""
    R = ref_lib()
    if R is None:
        return None
    px = np.ascontiguousarray(x, np.float64)
    py = np.ascontiguousarray(y, np.float64)
    q = np.ones(len(px))
    fx, fy = np.zeros(len(px)), np.zeros(len(px))
    R.bh_ref_forces_sample(len(px), _p(px, C.c_double), _p(py, C.c_double),
                           _p(q, C.c_double), theta, k, min_dist, _p(fx, C.c_double),
                           _p(fy, C.c_double), threads, stride)
    return fx, fy


# ---- DCT Poisson density, FP64 (force_electrostatic.py) --------------------
def density_bins(x, y, die_w, die_h, G):
    """Point-in-bin (force_electrostatic.py:55-56) with the division in f32."""
    bw = np.float32(die_w) / np.float32(G)
    bh = np.float32(die_h) / np.float32(G)

    def one(v, b):
        q = _f32(v) / b
        out = np.zeros(len(q), np.int64)
        ok = q >= 1.0
        out[ok] = np.minimum(np.floor(q[ok]).astype(np.int64), G - 1)
        out[q >= np.float32(G - 1)] = G - 1
        return out
    return one(x, bw), one(y, bh), float(bw), float(bh)


def density_map(x, y, area, die_w, die_h, G):
    """rho[r, c] += area / (bw * bh) (force_electrostatic.py:47-60), FP64."""
    col, row, bw, bh = density_bins(x, y, die_w, die_h, G)
    rho = np.zeros((G, G))
    np.add.at(rho, (row, col), np.asarray(area, np.float64) / (bw * bh))
    return rho, col, row, bw, bh


def solve_poisson(rho, wx, wy):
    """_solve_poisson_fft (force_electrostatic.py:62-105) in FP64."""
    from scipy.fft import dctn, idctn
    rho_hat = dctn(rho, type=2, norm="ortho")
    ny, nx = rho.shape
    kx, ky = np.meshgrid(np.arange(nx), np.arange(ny))
    eig = (wx * np.cos(np.pi * kx / nx) - wx) ** 2 + (wy * np.cos(np.pi * ky / ny) - wy) ** 2
    eig[0, 0] = 1.0
    phi_hat = -rho_hat / eig
    phi_hat[0, 0] = 0.0
    phi = idctn(phi_hat, type=2, norm="ortho")
    ex = np.zeros_like(phi)
    ey = np.zeros_like(phi)
    ex[:, 1:-1] = -(phi[:, 2:] - phi[:, :-2]) * wx * 0.5
    ey[1:-1, :] = -(phi[2:, :] - phi[:-2, :]) * wy * 0.5
    ex[:, 0] = -(phi[:, 1] - phi[:, 0]) * wx
    ex[:, -1] = -(phi[:, -1] - phi[:, -2]) * wx
    ey[0, :] = -(phi[1, :] - phi[0, :]) * wy
    ey[-1, :] = -(phi[-1, :] - phi[-2, :]) * wy
    return phi, ex, ey


def density_forces(x, y, area, die_w, die_h, G, target=0.7, weight=1.0):
    """ElectrostaticSmoothingForce.calculate (force_electrostatic.py:107-157)."""
    rho, col, row, bw, bh = density_map(x, y, area, die_w, die_h, G)
    charge = rho - target
    phi, ex, ey = solve_poisson(charge, 1.0 / bw, 1.0 / bh)
    q = np.asarray(area, np.float64)
    fx = q * ex[row, col] * weight
    fy = q * ey[row, col] * weight
    energy = float(np.sum(0.5 * q * phi[row, col]) * weight)
    return dict(fx=fx, fy=fy, rho=charge, phi=phi, ex=ex, ey=ey, energy=energy)


# ---- the composite plain iteration ------------------------------------------
def plain_forces(adj_ptr, adj_idx, x, y, area, die_w, die_h, k=1.0, repel=0.5, theta=0.5,
                 min_dist=0.1, bins=0, target=0.7, weight=0.0, threads=1):
    """Total force of one plain iteration at positions (x, y): attraction
    (placer.rs:243-255 over the full adjacency) + Barnes-Hut repulsion (law of
    placer.rs:258-272, tree rules of BarnesHutTree.cpp) + the DCT Poisson
    density force (force_electrostatic.py:107-157) when bins > 0.

    Returns f64 = (fx, fy), the FP64 recomputation (Barnes-Hut over each
    point's interaction list), and f32 = (fx, fy), the same sum in f32 in
    the device's order ((attraction + Barnes-Hut) + (area * E) * weight) with
    the field taken from the FP64 solve and rounded once to f32."""
    x, y = _f32(x), _f32(y)
    a64 = attraction_f64(adj_ptr, adj_idx, x, y, k)
    a32 = attraction_f32(adj_ptr, adj_idx, x, y, k)
    fx64, fy64 = np.array(a64[0], np.float64), np.array(a64[1], np.float64)
    fx32, fy32 = a32[0].astype(np.float32), a32[1].astype(np.float32)
    if repel != 0.0:
        b = bh_forces(x, y, repel, theta, min_dist, threads=threads)
        fx64 += b["fx"]
        fy64 += b["fy"]
        fx32 = (fx32 + b["fx32"]).astype(np.float32)
        fy32 = (fy32 + b["fy32"]).astype(np.float32)
    if bins > 0 and weight != 0.0:
        d = density_forces(x, y, area, die_w, die_h, bins, target, weight)
        fx64 += d["fx"]
        fy64 += d["fy"]
        col, row, _, _ = density_bins(x, y, die_w, die_h, bins)
        q = np.asarray(area, np.float32)
        w = np.float32(weight)
        ex = d["ex"][row, col].astype(np.float32)
        ey = d["ey"][row, col].astype(np.float32)
        fx32 = (fx32 + (q * ex).astype(np.float32) * w).astype(np.float32)
        fy32 = (fy32 + (q * ey).astype(np.float32) * w).astype(np.float32)
    return dict(f64=(fx64, fy64), f32=(fx32, fy32))


def plain_run(adj_ptr, adj_idx, x0, y0, area, die_w, die_h, iters, dt=0.1, damping=0.9,
              **force_kw):
    """`iters` plain iterations from (x0, y0) at rest: the f32 forces of
    plain_forces, then the damped step clamped to the die (placer.rs:275-280).
    Returns the final positions."""
    x, y = _f32(x0).copy(), _f32(y0).copy()
    vx, vy = np.zeros_like(x), np.zeros_like(y)
    for _ in range(iters):
        fx, fy = plain_forces(adj_ptr, adj_idx, x, y, area, die_w, die_h, **force_kw)["f32"]
        integrate(x, y, vx, vy, fx, fy, dt, damping, (0.0, 0.0, die_w, die_h))
    return x, y


# ---- attention scores (attention.rs, hierarchy.rs) -------------------------
def hierarchy_nodes(leaf_ptr, leaf_gate, leaf_depth):
    """The explicit binary tree of a hierarchy from its leaves in DFS order and
    their depths (every internal node of recursive_bisect has two children,
    partitioner.rs:85-99): a list of (depth, gates) for every node, in DFS
    preorder. Internal nodes hold the union of their leaves' gates."""
    leaf_ptr, leaf_gate, leaf_depth = list(leaf_ptr), list(leaf_gate), list(leaf_depth)
    nodes = []
    pos = [0]

    def parse(depth):
        i = pos[0]
        if i >= len(leaf_depth):
            raise ValueError("leaf depths do not form a full binary tree")
        slot = len(nodes)
        nodes.append(None)
        if leaf_depth[i] == depth:
            pos[0] += 1
            gates = leaf_gate[leaf_ptr[i]:leaf_ptr[i + 1]]
        elif leaf_depth[i] > depth:
            gates = parse(depth + 1) + parse(depth + 1)
        else:
            raise ValueError("leaf depths do not form a full binary tree")
        nodes[slot] = (depth, gates)
        return gates

    if leaf_depth:
        parse(0)
        if pos[0] != len(leaf_depth):
            raise ValueError("leaf depths do not form a full binary tree")
    return nodes


def clusters_at_depth(nodes, depth):
    """HierarchyTree::clusters_at_depth (hierarchy.rs:134-159): the nodes at
    `depth` in DFS order (preorder lists them in that order)."""
    return [g for d, g in nodes if d == depth]


def attention_level(net_ptr, net_gate, clusters, top_k=10):
    """compute_level_attention (attention.rs:50-88) literally, with
    nets_touching_gates (:90-99) as Python sets: scores[n][n] f32 and the
    top_k lists. For small cases."""
    net_ptr, net_gate = list(net_ptr), list(net_gate)
    m = len(net_ptr) - 1
    n = len(clusters)
    nets = []
    for gates in clusters:
        gs = set(int(g) for g in gates)
        nets.append({e for e in range(m)
                     if any(g in gs for g in net_gate[net_ptr[e]:net_ptr[e + 1]])})
    scores = np.zeros((n, n), np.float32)
    for i in range(n):
        total = len(nets[i])
        if total == 0:
            continue
        for j in range(n):
            if i != j:
                scores[i, j] = np.float32(len(nets[i] & nets[j])) / np.float32(total)
    tops = []
    for i in range(n):
        idx = sorted((j for j in range(n) if j != i), key=lambda j: -scores[i, j])
        tops.append([j for j in idx[:top_k] if scores[i, j] > 0])
    return scores, tops


def attention_all(net_ptr, net_gate, leaf_ptr, leaf_gate, leaf_depth, top_k=10):
    """compute_all_attention (attention.rs:33-48): one (depth, scores, top_k)
    per depth with at least two clusters."""
    nodes = hierarchy_nodes(leaf_ptr, leaf_gate, leaf_depth)
    out = []
    for depth in range(max((d for d, _ in nodes), default=-1) + 1):
        cl = clusters_at_depth(nodes, depth)
        if len(cl) >= 2:
            s, t = attention_level(net_ptr, net_gate, cl, top_k)
            out.append((depth, s, t))
    return out


def attention_level_sparse(net_ptr, net_gate, n_gates, cluster_ptr, cluster_gate, top_k=10):
    """The same level as attention_level, vectorised for large cases with a
    sparse cluster-by-net incidence matrix B (scipy.sparse): shared = B B^T,
    totals = row sums of B. Returns the nonzero off-diagonal scores as
    (rows, cols, f32 scores) sorted by (row, col) and the top_k lists padded
    with -1 to [n, top_k]."""
    import scipy.sparse as sp

    net_ptr, net_gate = np.asarray(net_ptr, np.int64), np.asarray(net_gate, np.int64)
    cluster_ptr = np.asarray(cluster_ptr, np.int64)
    n = len(cluster_ptr) - 1
    m = len(net_ptr) - 1
    cl = np.full(n_gates, -1, np.int64)
    cl[np.asarray(cluster_gate, np.int64)] = np.repeat(np.arange(n), np.diff(cluster_ptr))
    pin_net = np.repeat(np.arange(m), np.diff(net_ptr))
    pin_cl = cl[net_gate]
    keep = pin_cl >= 0
    B = sp.csr_matrix((np.ones(int(keep.sum()), np.int64), (pin_cl[keep], pin_net[keep])),
                      shape=(n, m))
    B.sum_duplicates()
    B.data[:] = 1  # a net touching a cluster through several pins counts once
    total = np.asarray(B.sum(axis=1)).ravel()
    S = (B @ B.T).tocoo()
    off = S.row != S.col
    r, c, v = S.row[off].astype(np.int64), S.col[off].astype(np.int64), S.data[off]
    o = np.lexsort((c, r))
    r, c, v = r[o], c[o], v[o]
    sc = v.astype(np.float32) / total[r].astype(np.float32)
    tk = np.full((n, max(top_k, 0)), -1, np.int32)
    if top_k > 0 and len(r):
        o = np.lexsort((c, -sc.astype(np.float64), r))
        rr, cc = r[o], c[o]
        start = np.searchsorted(rr, np.arange(n))
        rank = np.arange(len(rr)) - start[rr]
        sel = rank < top_k
        tk[rr[sel], rank[sel]] = cc[sel]
    return r, c, sc, tk


def attention_sample(net_ptr, net_gate, cluster_ptr, cluster_gate, rows, top_k=10):
    """The C++ restatement of compute_level_attention on the sampled clusters
    `rows` of one level (all of them for the whole level): (scores among the
    samples [k, k], top_k lists [k, top_k] -1 padded, seconds of the net-set,
    intersection and top-k phases)."""
    net_ptr, net_gate = _i32(net_ptr), _i32(net_gate)
    cp, cg, rows = _i32(cluster_ptr), _i32(cluster_gate), _i32(rows)
    k = len(rows)
    sc = np.zeros((k, k), np.float32)
    tk = np.full((k, max(top_k, 1)), -1, np.int32)
    t = np.zeros(3, np.float64)
    lib().or_attention_sample(len(net_ptr) - 1, _p(net_ptr, C.c_int32), _p(net_gate, C.c_int32),
                              len(cp) - 1, _p(cp, C.c_int32), _p(cg, C.c_int32), k,
                              _p(rows, C.c_int32), top_k, _p(sc, C.c_float),
                              _p(tk, C.c_int32), _p(t, C.c_double))
    return sc, tk[:, :top_k], t

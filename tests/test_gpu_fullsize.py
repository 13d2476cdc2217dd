"""Parity at the full plain-1M size (1,000,000 gates, 1,200,000 nets, die
1200 x 1200, 512 x 512 congestion, DCT 1024 x 1024): every stage against the
oracle on the whole netlist. The literal congestion loop is O(sum of bounding
box areas), so the counts are checked against the oracle's difference-array
restatement of it (tested against the literal loop on the CPU); Barnes-Hut
runs the oracle's walk on all host threads."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32_01 = float(np.float32(0.1))


@pytest.fixture(scope="module")
def full(fx):
    return fx.synth_plain(42, 1_000_000, 1_200_000, 1200.0)


@pytest.fixture(scope="module")
def full_design(fx, ctx, full):
    d = fx.Design(ctx, full.circuit)
    yield d
    d.close()


def _rel(ax, ay, bx, by):
    num = np.sqrt(((np.asarray(ax, np.float64) - bx) ** 2 + (np.asarray(ay, np.float64) - by) ** 2).sum())
    return num / np.sqrt((np.asarray(bx, np.float64) ** 2 + np.asarray(by, np.float64) ** 2).sum())


def test_congestion_and_hpwl(full_design, full, oracle):
    c, p = full.circuit, full.placement
    counts, hpwl, tot, mx = full_design.congestion(512, 512, p.gate_x, p.gate_y)
    want = oracle.congestion_counts(c.net_ptr, c.net_gate, p.gate_x, p.gate_y,
                                    c.chip_width, c.chip_height, 512, 512)
    assert np.array_equal(counts, want)
    ref = oracle.hpwl_f64(c.net_ptr, c.net_gate, p.gate_x, p.gate_y)
    assert abs(hpwl - ref) <= 1e-12 * ref
    _, _, cap = oracle.grid_geometry(c.chip_width, c.chip_height, 512, 512)
    h = want.astype(np.float32)
    rt, rm = oracle.overflow(h, h, 512, 512, cap)
    assert mx == rm and abs(tot - rt) <= 5e-3 * max(rt, 1.0)


def test_adjacency_and_attraction(full_design, full, oracle):
    c, p = full.circuit, full.placement
    ap, ai = full_design.adjacency()
    rp, ri = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    assert np.array_equal(ap, rp) and np.array_equal(ai, ri)
    full_design.set_positions(p.gate_x, p.gate_y)
    fx_, fy_ = full_design.attraction(1.0)
    ox, oy = oracle.attraction_f32(rp, ri, p.gate_x, p.gate_y, 1.0)
    assert np.array_equal(fx_, ox) and np.array_equal(fy_, oy)
    dx, dy = oracle.attraction_f64(rp, ri, p.gate_x, p.gate_y, 1.0)
    assert _rel(fx_, fy_, dx, dy) < 1e-5


def test_barnes_hut_and_one_plain_iteration(fx, full_design, full, oracle):
    """Keys, sort order and forces of all 1M points bit-exact; then one plain
    iteration (attraction + Barnes-Hut + damped step, density off) ends on the
    oracle's positions, and the congestion of those positions matches."""
    c, p = full.circuit, full.placement
    d = full_design
    d.set_positions(p.gate_x, p.gate_y)
    bx, by, keys, perm, root = d.barnes_hut(0.5, 0.5, 0.1)
    o = oracle.bh_forces(p.gate_x, p.gate_y, 0.5, 0.5, F32_01, threads=os.cpu_count() or 1)
    assert np.array_equal(root, o["root"])
    assert np.array_equal(keys, o["keys"]) and np.array_equal(perm, o["perm"])
    assert np.array_equal(bx, o["fx32"]) and np.array_equal(by, o["fy32"])
    assert _rel(bx, by, o["fx"], o["fy"]) < 1e-5
    cfg = fx.iter_cfg(density_bins=0, cong_cols=512, cong_rows=512, bh_walk=fx.FX_BH_EXACT)
    x, y = p.gate_x.copy(), p.gate_y.copy()
    st = d.force_iterate(cfg, 1, x, y)
    rp, ri = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    ax, ay = oracle.attraction_f32(rp, ri, p.gate_x, p.gate_y, 1.0)
    ox, oy = p.gate_x.copy(), p.gate_y.copy()
    vx, vy = np.zeros_like(ox), np.zeros_like(oy)
    oracle.integrate(ox, oy, vx, vy, ax + o["fx32"], ay + o["fy32"], 0.1, 0.9,
                     (0.0, 0.0, c.chip_width, c.chip_height))
    assert np.array_equal(x, ox) and np.array_equal(y, oy)
    want = oracle.congestion_counts(c.net_ptr, c.net_gate, ox, oy, c.chip_width,
                                    c.chip_height, 512, 512)
    counts, hpwl, _, _ = d.congestion(512, 512)
    assert np.array_equal(counts, want)
    assert hpwl == st.hpwl
    assert abs(hpwl - oracle.hpwl_f64(c.net_ptr, c.net_gate, ox, oy)) <= 1e-12 * hpwl


@pytest.mark.parametrize("prec", ["simt", "i8"])
def test_density_field_and_forces(fx, full_design, full, oracle, prec):
    """The 1024 x 1024 solve of the 1M-gate workload within 1e-5 of the FP64
    FFT oracle: FP32 GEMMs on the CUDA cores, and on the tensor cores from
    exact 8-bit slices."""
    c, p = full.circuit, full.placement
    full_design.set_positions(p.gate_x, p.gate_y)
    code = {"simt": fx.FX_DCT_SIMT, "i8": fx.FX_DCT_I8}[prec]
    out = full_design.density(1024, 0.7, 1.0, code, grids=True)
    area = (c.gate_widths * c.gate_heights).astype(np.float64)
    ref = oracle.density_forces(p.gate_x, p.gate_y, area, c.chip_width, c.chip_height, 1024,
                                0.7, 1.0)
    fe = _rel(out["ex"], out["ey"], ref["ex"], ref["ey"])
    ff = _rel(out["fx"], out["fy"], ref["fx"], ref["fy"])
    print(f"density 1M G=1024 {prec}: field {fe:.3e} force {ff:.3e}")
    assert fe < 1e-5 and ff < 1e-5


@pytest.mark.parametrize("weight,iters", [(1e-4, 3), (1.0, 1)])
def test_benchmarked_step_with_density(fx, ctx, full, oracle, weight, iters):
    """The bench's step at full size: attraction + Barnes-Hut + DCT density
    (1024 x 1024, FP32) + damped step + 512 x 512 congestion, checked by the
    same rules as the 20k-gate case (test_gpu_parity._step_parity): the last
    iteration's total force within 1e-5 of FP64, its step bit for bit, the
    final congestion counts bit-exact, HPWL and overflow of the run within
    0.5 % of the oracle's run."""
    from test_gpu_parity import _step_parity
    _step_parity(fx, ctx, oracle, full, 1024, weight, iters, (512, 512),
                 threads=os.cpu_count() or 1)


def test_hierarchy(fx, full_design, full, oracle):
    c = full.circuit
    tree = full_design.partition(fx.part_cfg())
    ap, ai = full_design.adjacency()
    ot = oracle.build_hierarchy(c.num_gates, ap, ai, c.chip_width, c.chip_height)
    assert np.array_equal(tree["leaf_ptr"], ot["leaf_ptr"])
    assert np.array_equal(tree["leaf_gate"], ot["leaf_gate"])
    assert np.array_equal(tree["leaf_depth"], ot["leaf_depth"])
    assert tree["num_nodes"] == ot["num_nodes"]


def test_leaf_batch_full_size(fx, ctx, oracle):
    """The batched-leaf workload in full: 16,384 clusters of 16-128 gates, 300
    iterations, autotuned schedule; every gate bit-identical to the oracle's
    place_gates_in_leaf, run leaf by leaf on all host threads."""
    from concurrent.futures import ThreadPoolExecutor
    s = fx.synth_leaves(42, 16_384, 16, 128, 1.5)
    c = s.circuit
    gates = np.arange(c.num_gates, dtype=np.int32)
    d = fx.Design(ctx, c)
    try:
        x, y, _ = d.place_leaves(s.leaf_ptr, gates, s.region, fx.leaf_cfg(force_iterations=300))
    finally:
        d.close()
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    ox = np.zeros(c.num_gates, np.float32)
    oy = np.zeros(c.num_gates, np.float32)
    lp, reg = s.leaf_ptr, s.region.reshape(-1, 4)

    def one(l):  # ctypes releases the GIL during the call
        oracle.place_leaf(gates[lp[l]:lp[l + 1]], ap, ai, reg[l], 300, 1.0, 0.5, 0.9, 0.1,
                          ox, oy)

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        list(ex.map(one, range(len(lp) - 1)))
    assert np.array_equal(x, ox) and np.array_equal(y, oy)


def test_leaf_batch_fast_precision_full_size(fx, ctx, oracle):
    """FX_LEAF_FAST on the whole batched-leaf workload (16,384 clusters,
    300 iterations): the first iteration's total force of every gate within
    1e-5 (relative L2) of the FP64 recomputation at the leaves' start
    positions, and the final HPWL within 0.5 % of place_gates_in_leaf's."""
    from concurrent.futures import ThreadPoolExecutor
    s = fx.synth_leaves(42, 16_384, 16, 128, 1.5)
    c = s.circuit
    gates = np.arange(c.num_gates, dtype=np.int32)
    d = fx.Design(ctx, c)
    try:
        d.trace(True)
        x, y, _ = d.place_leaves(s.leaf_ptr, gates, s.region,
                                 fx.leaf_cfg(force_iterations=300, precision=fx.FX_LEAF_FAST))
        tfx, tfy = d.leaf_trace_get(c.num_gates)
        ix, iy, _ = d.place_leaves(s.leaf_ptr, gates, s.region,
                                   fx.leaf_cfg(force_iterations=300))
        efx, efy = d.leaf_trace_get(c.num_gates)
    finally:
        d.close()
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    lp, reg = s.leaf_ptr, s.region.reshape(-1, 4)
    x0 = np.zeros(c.num_gates, np.float32)
    y0 = np.zeros(c.num_gates, np.float32)
    rfx = np.zeros(c.num_gates)
    rfy = np.zeros(c.num_gates)
    ox = np.zeros(c.num_gates, np.float32)
    oy = np.zeros(c.num_gates, np.float32)

    def one(l):
        g = gates[lp[l]:lp[l + 1]]
        oracle.place_leaf(g, ap, ai, reg[l], 0, 1.0, 0.5, 0.9, 0.1, x0, y0)  # start positions
        rfx[g], rfy[g] = oracle.leaf_forces_f64(g, ap, ai, x0[g], y0[g])
        oracle.place_leaf(g, ap, ai, reg[l], 300, 1.0, 0.5, 0.9, 0.1, ox, oy)

    with ThreadPoolExecutor(os.cpu_count() or 1) as ex:
        list(ex.map(one, range(len(lp) - 1)))
    err_fast = _rel(tfx, tfy, rfx, rfy)
    err_ieee = _rel(efx, efy, rfx, rfy)
    print(f"leaf forces vs FP64: fast {err_fast:.3e}, IEEE {err_ieee:.3e}")
    assert err_fast <= 1e-5 and err_ieee <= 1e-5
    assert np.array_equal(ix, ox) and np.array_equal(iy, oy)  # IEEE: bit-exact
    h_fast = oracle.hpwl_f64(c.net_ptr, c.net_gate, x, y)
    h_ref = oracle.hpwl_f64(c.net_ptr, c.net_gate, ox, oy)
    print(f"leaf HPWL: fast {h_fast:.6e} vs reference {h_ref:.6e}")
    assert abs(h_fast - h_ref) <= 5e-3 * h_ref

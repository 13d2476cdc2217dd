"""Parity of the CUDA hot path with the CPU oracle (runs on a B200).

Bars: integer/index work bit-exact; forces within 1e-5 relative (global L2)
of an FP64 recomputation on the same positions; final HPWL/overflow of a run
within 0.5 % of the oracle's run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32_01 = float(np.float32(0.1))  # the device's f32 min_dist, exactly
FX_BH_FAST = 0  # fx_iter_cfg.bh_walk / fx_stage_barnes_hut_walk: hardware rsqrt
FX_BH_EXACT = 1  # per-point walk, bit-identical to the oracle's f32 order


def rel_l2(ax, ay, bx, by):
    return float(np.sqrt(((ax - bx) ** 2 + (ay - by) ** 2).sum() /
                         max((bx ** 2 + by ** 2).sum(), 1e-300)))


@pytest.fixture(scope="module")
def small_design(fx, ctx, plain_small):
    d = fx.Design(ctx, plain_small.circuit)
    d.set_positions(plain_small.placement.gate_x, plain_small.placement.gate_y)
    yield d
    d.close()


# ---- rows D + F --------------------------------------------------------------
@pytest.mark.parametrize("cols,rows", [(64, 64), (37, 53), (1, 1), (256, 256), (512, 7)])
def test_congestion_bit_exact(small_design, plain_small, oracle, cols, rows):
    c, p = plain_small.circuit, plain_small.placement
    counts, hpwl, tot, mx = small_design.congestion(cols, rows)
    h, v = oracle.congestion(c.net_ptr, c.net_gate, p.gate_x, p.gate_y,
                             c.chip_width, c.chip_height, cols, rows)
    assert np.array_equal(counts.astype(np.float32), h)
    assert np.array_equal(h, v)
    ref = oracle.hpwl_f64(c.net_ptr, c.net_gate, p.gate_x, p.gate_y)
    assert abs(hpwl - ref) <= 1e-12 * ref
    _, _, cap = oracle.grid_geometry(c.chip_width, c.chip_height, cols, rows)
    rt, rm = oracle.overflow(h, v, cols, rows, cap)
    assert mx == rm
    ov = np.maximum((h + v) - np.float32(cap), np.float32(0)).astype(np.float64)
    assert abs(tot - ov.sum()) <= 1e-12 * max(ov.sum(), 1.0)  # FP64 recomputation
    assert abs(tot - rt) <= 5e-3 * max(rt, 1.0)  # the reference's f32 running sum
    # the reference's own f32 running sum stays within 0.5 %
    assert abs(hpwl - oracle.hpwl_f32(c.net_ptr, c.net_gate, p.gate_x, p.gate_y)) <= 5e-3 * ref


def test_congestion_edge_cases(fx, ctx, oracle):
    # empty and single-pin nets (skipped), a gate named twice, positions below
    # zero / beyond the die / on cell boundaries / NaN, and a net whose every
    # position is NaN (min > max: no cells).
    nets = [[], [3], [0, 0], [1, 2, 3], [4, 5], [6, 7], [8, 9], [0, 9, 5], [10, 11]]
    circ = fx.Circuit.from_nets(nets, 12, chip_width=100.0, chip_height=100.0)
    x = np.array([10, -5, 250, 20, 30, 40, np.nan, 50, 1e30, 0.0, np.nan, np.nan], np.float32)
    y = np.array([10, 50, 60, -1e30, 12.5, 25, 5, np.nan, 99.99, 100, np.nan, np.nan],
                 np.float32)
    d = fx.Design(ctx, circ)
    try:
        for cols, rows in ((8, 8), (10, 10), (3, 17)):
            counts, hpwl, tot, mx = d.congestion(cols, rows, x, y)
            h, v = oracle.congestion(circ.net_ptr, circ.net_gate, x, y, 100.0, 100.0,
                                     cols, rows)
            assert np.array_equal(counts.astype(np.float32), h)
    finally:
        d.close()


def test_congestion_repeat_calls_are_identical(small_design):
    a = small_design.congestion(64, 64)
    b = small_design.congestion(64, 64)
    assert np.array_equal(a[0], b[0]) and a[1:] == b[1:]


def test_reference_api_build_and_compute(fx, plain_small, oracle):
    c, p = plain_small.circuit, plain_small.placement
    g = fx.build_and_compute(p, c, 64, 64)
    h, _ = oracle.congestion(c.net_ptr, c.net_gate, p.gate_x, p.gate_y,
                             c.chip_width, c.chip_height, 64, 64)
    assert np.array_equal(g.h_congestion, h) and np.array_equal(g.v_congestion, h)


# ---- row A ---------------------------------------------------------------------
def test_adjacency_matches_reference(small_design, plain_small, oracle):
    c = plain_small.circuit
    ap, ai = small_design.adjacency()
    rp, ri = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    assert np.array_equal(ap, rp)
    for g in range(0, c.num_gates, 7):
        assert sorted(ai[ap[g]:ap[g + 1]]) == sorted(ri[rp[g]:rp[g + 1]])


def test_adjacency_order_is_reference_order(small_design, plain_small, oracle):
    c = plain_small.circuit
    ap, ai = small_design.adjacency()
    rp, ri = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    assert np.array_equal(ap, rp) and np.array_equal(ai, ri)


def test_attraction_bit_exact_and_vs_fp64(small_design, plain_small, oracle):
    p, c = plain_small.placement, plain_small.circuit
    rp, ri = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    fx_, fy_ = small_design.attraction(1.0)
    sx, sy = oracle.attraction_f32(rp, ri, p.gate_x, p.gate_y, 1.0)
    assert np.array_equal(fx_, sx) and np.array_equal(fy_, sy)  # reference f32 order
    rx, ry = oracle.attraction_f64(rp, ri, p.gate_x, p.gate_y, 1.0)
    assert rel_l2(fx_, fy_, rx, ry) < 1e-5


# ---- row B ---------------------------------------------------------------------
def _bh_check(d, x, y, oracle, k=0.5, theta=0.5):
    d.set_positions(x, y)
    bx, by, keys, perm, root = d.barnes_hut(k, theta, 0.1)
    o = oracle.bh_forces(x, y, k, theta, F32_01)
    assert np.array_equal(root, o["root"])
    assert np.array_equal(keys, o["keys"])  # Morton keys bit-exact
    assert np.array_equal(perm, o["perm"])  # stable sort order exact
    assert np.array_equal(bx, o["fx32"]) and np.array_equal(by, o["fy32"])  # bit-exact
    assert rel_l2(bx, by, o["fx"], o["fy"]) < 1e-5  # FP64, same interaction list
    # the hardware-rsqrt walk: the same tree, the same interaction count per
    # point, forces within f32 rounding
    qx, qy, qkeys, qperm, qroot, terms = d.barnes_hut(k, theta, 0.1, walk=FX_BH_FAST,
                                                      terms=True)
    assert np.array_equal(qkeys, keys) and np.array_equal(qperm, perm)
    assert np.array_equal(terms, o["interactions"])
    assert rel_l2(qx, qy, o["fx"], o["fy"]) < 1e-5
    assert rel_l2(qx, qy, o["fx32"].astype(np.float64), o["fy32"].astype(np.float64)) < 1e-5
    return bx, by


def test_barnes_hut_config1(small_design, plain_small, oracle):
    p = plain_small.placement
    bx, by = _bh_check(small_design, p.gate_x, p.gate_y, oracle)
    ref = oracle.bh_reference(p.gate_x, p.gate_y, 0.5, 0.5, 0.1)
    if ref is not None:  # the reference's own tree, when built here
        assert rel_l2(bx, by, *ref) < 5e-3


@pytest.mark.parametrize("case", ["coincident", "pair", "line", "clumps", "tiny"])
def test_barnes_hut_degenerate(fx, ctx, oracle, case):
    rng = np.random.default_rng(3)
    n = {"coincident": 300, "pair": 2, "line": 2000, "clumps": 5000, "tiny": 3}[case]
    if case == "coincident":
        x = np.full(n, 7.25, np.float32); y = np.full(n, 3.5, np.float32)
    elif case == "pair":
        x = np.array([1.0, 1.05], np.float32); y = np.array([2.0, 2.0], np.float32)
    elif case == "line":
        x = np.linspace(0, 50, n).astype(np.float32); y = np.full(n, 10.0, np.float32)
    elif case == "clumps":
        c = rng.integers(0, 20, n)
        x = (c * 5.0 + rng.integers(0, 3, n) * 1e-3).astype(np.float32)
        y = (c * 2.0).astype(np.float32)
    else:
        x = np.array([0.0, 1e-6, 2e-6], np.float32); y = np.zeros(3, np.float32)
    circ = fx.Circuit.from_nets([[0, 1]] if n >= 2 else [], n, 100.0, 100.0)
    d = fx.Design(ctx, circ)
    try:
        bx, by = _bh_check(d, x, y, oracle)
        assert np.all(np.isfinite(bx)) and np.all(np.isfinite(by))
    finally:
        d.close()


def test_barnes_hut_clustered_large(fx, ctx, oracle):
    rng = np.random.default_rng(5)
    n = 200_000
    centers = rng.random((50, 2)) * 1000
    pick = rng.integers(0, 50, n)
    pts = (centers[pick] + rng.normal(0, 8.0, (n, 2))).astype(np.float32)
    circ = fx.Circuit.from_nets([[0, 1]], n, 1200.0, 1200.0)
    d = fx.Design(ctx, circ)
    try:
        _bh_check(d, pts[:, 0].copy(), pts[:, 1].copy(), oracle)
    finally:
        d.close()


# ---- row C ---------------------------------------------------------------------
# Relative L2 error bars of the potential / field / force against the FP64
# FFT oracle, per GEMM precision: FP32 CUDA-core GEMMs, 3xTF32 and single-pass
# TF32 / BF16 tensor-core GEMMs (all accumulate in FP32).
# "3xtf32" (FX_DCT_FP32) is the tensor-core split: FP32 inputs, but its error
# grows with G (the accumulation on the tensor cores); "simt" is FP32 on the
# CUDA cores, the iteration's default.
# "i8" (FX_DCT_I8) is the tensor-core path from exact 8-bit slices with
# integer accumulation: FP32-accurate at every G.
PREC_TOL = {"simt": (1e-5, 2e-5), "3xtf32": (2e-4, 2e-4), "tf32": (1e-2, 1e-2),
            "bf16": (5e-2, 5e-2), "i8": (1e-5, 1e-5)}


@pytest.mark.parametrize("G", [128, 256])
@pytest.mark.parametrize("prec", ["simt", "i8", "3xtf32", "tf32", "bf16"])
def test_density_vs_fp64(fx, ctx, oracle, G, prec):
    s = fx.synth_plain(9, 20_000, 24_000, 170.0)
    c, p = s.circuit, s.placement
    code = {"simt": fx.FX_DCT_SIMT, "3xtf32": fx.FX_DCT_FP32, "tf32": fx.FX_DCT_TF32,
            "bf16": fx.FX_DCT_BF16, "i8": fx.FX_DCT_I8}[prec]
    tol_phi, tol_e = PREC_TOL[prec]
    d = fx.Design(ctx, c)
    try:
        d.set_positions(p.gate_x, p.gate_y)
        out = d.density(G, 0.7, 1.0, code, grids=True)
        area = (c.gate_widths * c.gate_heights).astype(np.float64)
        ref = oracle.density_forces(p.gate_x, p.gate_y, area, c.chip_width, c.chip_height,
                                    G, 0.7, 1.0)
        assert np.allclose(out["rho"], ref["rho"], rtol=0, atol=1e-5)
        phi_err = np.linalg.norm(out["phi"] - ref["phi"]) / np.linalg.norm(ref["phi"])
        e_err = rel_l2(out["ex"].ravel(), out["ey"].ravel(), ref["ex"].ravel(), ref["ey"].ravel())
        f_err = rel_l2(out["fx"], out["fy"], ref["fx"], ref["fy"])
        print(f"density G={G} {prec}: phi {phi_err:.3e} field {e_err:.3e} force {f_err:.3e}")
        assert phi_err < tol_phi, phi_err
        assert e_err < tol_e, e_err
        assert f_err < tol_e
        assert abs(out["energy"] - ref["energy"]) <= 10 * tol_phi * abs(ref["energy"])
    finally:
        d.close()


# ---- rows A+B+E+D+F: the plain-small run ------------------------------------------
def _oracle_run(oracle, c, x0, y0, iters, box):
    rp, ri = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    ox, oy = x0.copy(), y0.copy()
    vx, vy = np.zeros_like(ox), np.zeros_like(oy)
    for _ in range(iters):
        fa_x, fa_y = oracle.attraction_f32(rp, ri, ox, oy, 1.0)
        b = oracle.bh_forces(ox, oy, 0.5, 0.5, F32_01)
        oracle.integrate(ox, oy, vx, vy, fa_x + b["fx32"], fa_y + b["fy32"], 0.1, 0.9, box)
    return ox, oy


def test_plain_small_run_matches_oracle(fx, ctx, plain_small, oracle):
    """200 iterations of attraction (k=1) + Barnes-Hut (theta 0.5) + damped
    step on the 10k-gate netlist with 64 x 64 congestion: the device run and
    the oracle's run end on bit-identical positions, so HPWL and overflow
    agree exactly (the 0.5 % bar is met with zero error)."""
    c, p = plain_small.circuit, plain_small.placement
    iters = 200
    cfg = fx.iter_cfg(density_bins=0, cong_cols=64, cong_rows=64, bh_walk=FX_BH_EXACT)
    d = fx.Design(ctx, c)
    try:
        x = p.gate_x.copy(); y = p.gate_y.copy()
        st = d.force_iterate(cfg, iters, x, y)
        counts, hpwl, tot, mx = d.congestion(64, 64, x, y)
    finally:
        d.close()
    assert st.hpwl == hpwl and st.total_overflow == tot
    ox, oy = _oracle_run(oracle, c, p.gate_x, p.gate_y, iters, (0.0, 0.0, 120.0, 120.0))
    assert np.array_equal(x, ox) and np.array_equal(y, oy)
    h, v = oracle.congestion(c.net_ptr, c.net_gate, ox, oy, c.chip_width, c.chip_height, 64, 64)
    assert np.array_equal(counts.astype(np.float32), h)
    ref_hpwl = oracle.hpwl_f64(c.net_ptr, c.net_gate, ox, oy)
    assert abs(hpwl - ref_hpwl) <= 1e-12 * ref_hpwl
    _, _, cap = oracle.grid_geometry(c.chip_width, c.chip_height, 64, 64)
    rt, rm = oracle.overflow(h, v, 64, 64, cap)
    assert mx == rm and abs(tot - rt) <= 5e-3 * max(rt, 1.0)
    # the reference's own f32 HPWL of the same positions, within 0.5 %
    assert abs(hpwl - oracle.hpwl_f32(c.net_ptr, c.net_gate, ox, oy)) <= 5e-3 * ref_hpwl


def test_plain_iteration_is_deterministic(fx, ctx):
    """The full composite iteration (with the DCT density term) gives
    bit-identical positions when repeated."""
    s = fx.synth_plain(3, 30_000, 36_000, 208.0)
    cfg = fx.iter_cfg(density_bins=256, cong_cols=128, cong_rows=128)
    d = fx.Design(ctx, s.circuit)
    try:
        out = []
        for _ in range(2):
            x = s.placement.gate_x.copy(); y = s.placement.gate_y.copy()
            st = d.force_iterate(cfg, 12, x, y)
            out.append((x, y, st.hpwl, st.total_overflow, st.density_energy))
    finally:
        d.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2:] == out[1][2:]


def test_saved_state_restores_the_step(fx, ctx):
    """save_state / restore_state: an iteration from the restored state (with
    non-zero velocities) repeats the first one bit for bit, and restore
    without a save is rejected."""
    s = fx.synth_plain(5, 20_000, 24_000, 170.0)
    cfg = fx.iter_cfg(density_bins=128, cong_cols=64, cong_rows=64)
    d = fx.Design(ctx, s.circuit)
    try:
        with pytest.raises(fx.FluxionError):
            d.restore_state()
        d.set_positions(s.placement.gate_x, s.placement.gate_y)
        d.force_iterate(cfg, 2)        # velocities are non-zero from here on
        d.save_state()
        out = []
        for _ in range(2):
            d.restore_state()
            st = d.force_iterate(cfg, 3)
            x, y = d.get_positions()
            out.append((x, y, st.hpwl, st.total_overflow))
    finally:
        d.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2:] == out[1][2:]


def test_graph_replay_matches_eager_iterations(fx, ctx):
    """Runs of >= 8 iterations replay a captured CUDA graph of two iterations
    (stage timing off); with stage timing on every iteration is launched
    eagerly. Both give the same positions and statistics bit for bit."""
    s = fx.synth_plain(11, 30_000, 36_000, 208.0)
    cfg = fx.iter_cfg(density_bins=256, cong_cols=128, cong_rows=128)
    d = fx.Design(ctx, s.circuit)
    try:
        out = []
        for profiling in (False, True):
            ctx.set_profiling(profiling)
            x = s.placement.gate_x.copy(); y = s.placement.gate_y.copy()
            st = d.force_iterate(cfg, 21, x, y)
            out.append((x, y, st.hpwl, st.total_overflow, st.density_energy))
    finally:
        ctx.set_profiling(False)
        d.close()
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])
    assert out[0][2:] == out[1][2:]


# ---- the benchmarked step: A + B + C (DCT density) + E, then D + F -----------------
def _step_parity(fx, ctx, oracle, s, G, weight, iters, cong, threads=1, tol=1e-5):
    """Runs `iters` plain iterations with the density term on (the composite
    iteration the bench times; from the second iteration on, the density
    comes from the step kernel's own scatter of the positions it wrote) and
    checks the last one against the oracle:
    * its total per-gate force against the FP64 recomputation at the
      positions it started from (relative L2 <= tol), and against the
      oracle's f32 sum (field rounded once to f32);
    * its damped step, bit for bit, from the traced start state and force;
    * the congestion counts of the final positions, bit for bit;
    then the run's HPWL and overflow against the oracle's own run of the
    same iterations (within 0.5 %)."""
    c, p = s.circuit, s.placement
    cols, rows = cong
    cfg = fx.iter_cfg(density_bins=G, density_weight=weight, cong_cols=cols, cong_rows=rows)
    area = (c.gate_widths * c.gate_heights).astype(np.float32)
    d = fx.Design(ctx, c)
    try:
        d.trace(True)
        x, y = p.gate_x.copy(), p.gate_y.copy()
        st = d.force_iterate(cfg, iters, x, y)
        t = d.trace_get()
        counts, hpwl, tot, mx = d.congestion(cols, rows, x, y)
        ap, ai = d.adjacency()
    finally:
        d.close()
    f = oracle.plain_forces(ap, ai, t["x0"], t["y0"], area, c.chip_width, c.chip_height,
                            k=1.0, repel=0.5, theta=0.5, min_dist=F32_01, bins=G,
                            target=0.7, weight=weight, threads=threads)
    err64 = rel_l2(t["fx"].astype(np.float64), t["fy"].astype(np.float64), *f["f64"])
    err32 = rel_l2(t["fx"].astype(np.float64), t["fy"].astype(np.float64),
                   *(v.astype(np.float64) for v in f["f32"]))
    print(f"step G={G} w={weight} it={iters}: force vs FP64 {err64:.3e}, vs f32 oracle "
          f"{err32:.3e}")
    assert err64 <= tol, err64
    assert err32 <= tol, err32
    # the damped step of the traced iteration, bit for bit
    ox, oy = t["x0"].copy(), t["y0"].copy()
    ovx, ovy = t["vx0"].copy(), t["vy0"].copy()
    oracle.integrate(ox, oy, ovx, ovy, t["fx"], t["fy"], 0.1, 0.9,
                     (0.0, 0.0, c.chip_width, c.chip_height))
    assert np.array_equal(ox, x) and np.array_equal(oy, y)
    # congestion of the device's final positions: bit-exact counts
    want = oracle.congestion_counts(c.net_ptr, c.net_gate, x, y, c.chip_width, c.chip_height,
                                    cols, rows)
    assert np.array_equal(counts, want)
    assert hpwl == st.hpwl and tot == st.total_overflow
    # the oracle's own run: HPWL and overflow within 0.5 %
    rx, ry = oracle.plain_run(ap, ai, p.gate_x, p.gate_y, area, c.chip_width, c.chip_height,
                              iters, k=1.0, repel=0.5, theta=0.5, min_dist=F32_01, bins=G,
                              target=0.7, weight=weight, threads=threads)
    ref_hpwl = oracle.hpwl_f64(c.net_ptr, c.net_gate, rx, ry)
    rc = oracle.congestion_counts(c.net_ptr, c.net_gate, rx, ry, c.chip_width, c.chip_height,
                                  cols, rows).astype(np.float32)
    _, _, cap = oracle.grid_geometry(c.chip_width, c.chip_height, cols, rows)
    rt, _ = oracle.overflow(rc, rc, cols, rows, cap)
    print(f"  hpwl {st.hpwl:.6e} vs oracle {ref_hpwl:.6e}; overflow {st.total_overflow:.6e} "
          f"vs {rt:.6e}")
    assert abs(st.hpwl - ref_hpwl) <= 5e-3 * ref_hpwl
    assert abs(st.total_overflow - rt) <= 5e-3 * max(rt, 1.0)
    return err64


@pytest.mark.parametrize("G", [128, 256])
@pytest.mark.parametrize("weight", [1e-4, 1.0])
@pytest.mark.parametrize("iters", [1, 3])
def test_step_with_density_vs_oracle(fx, ctx, oracle, G, weight, iters):
    s = fx.synth_plain(9, 20_000, 24_000, 170.0)
    _step_parity(fx, ctx, oracle, s, G, weight, iters, (128, 128))

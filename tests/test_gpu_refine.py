"""Congestion refinement (HAPR_fluxion_v4/src/algorithm/refiner.rs:34-126)
against the oracle's literal restatement: same iterations, bit-identical
positions, identical final overflow."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("grid,iters,thr", [(64, 30, 1.0), (37, 25, 0.0), (128, 12, 5.0)])
def test_refine_bit_exact(fx, ctx, oracle, plain_small, grid, iters, thr):
    c, p = plain_small.circuit, plain_small.placement
    cfg = fx.refine_cfg(max_iterations=iters, grid_cols=grid, grid_rows=grid,
                        overflow_threshold=thr)
    d = fx.Design(ctx, c)
    try:
        x, y = p.gate_x.copy(), p.gate_y.copy()
        st, counts = d.refine(cfg, x, y, counts=True)
    finally:
        d.close()
    ox, oy, oit, ost = oracle.refine(c.net_ptr, c.net_gate, p.gate_x, p.gate_y,
                                     c.chip_width, c.chip_height, iters, 5.0, thr,
                                     grid, grid)
    assert st.iterations == oit
    assert np.array_equal(x, ox) and np.array_equal(y, oy)
    assert st.total_overflow == ost["total_overflow"]
    assert st.max_overflow == ost["max_overflow"]
    h, _ = oracle.congestion(c.net_ptr, c.net_gate, ox, oy, c.chip_width, c.chip_height,
                             grid, grid)
    assert np.array_equal(counts.astype(np.float32), h)
    assert abs(st.hpwl - ost["hpwl_f32"]) <= 5e-3 * st.hpwl


def test_refine_stops_when_uncongested(fx, ctx):
    # a single short net: overflow 0 <= threshold -> no iteration moves
    c = fx.Circuit.from_nets([[0, 1]], 3, 100.0, 100.0)
    d = fx.Design(ctx, c)
    try:
        x = np.array([10, 11, 50], np.float32); y = np.array([10, 10, 50], np.float32)
        st = d.refine(fx.refine_cfg(grid_cols=10, grid_rows=10), x, y)
    finally:
        d.close()
    assert st.iterations == 0 and st.moves == 0 and st.total_overflow == 0.0

"""Barnes-Hut deep keys on the device (row B): on dies where a level-15 cell
is not accepted by every point, the tree continues 12 levels below it. The
device must pick the same mode as the oracle from the same positions and
match it bit for bit, whether the host launched the deep kernels because the
die is large or because the positions were not known to lie in the die."""
import numpy as np
import pytest

from test_bh_deep_oracle import _crowded

pytestmark = pytest.mark.gpu

F32_01 = float(np.float32(0.1))


def _check(fx, ctx, oracle, x, y, chip):
    circ = fx.Circuit.from_nets([[0, 1]], len(x), chip, chip)
    d = fx.Design(ctx, circ)
    try:
        d.set_positions(x, y)
        bx, by, keys, perm, root = d.barnes_hut(0.5, 0.5, 0.1)
        bx2, by2, _, _, _ = d.barnes_hut(0.5, 0.5, 0.1)
        qx, qy, qkeys, _, _, terms = d.barnes_hut(0.5, 0.5, 0.1, walk=fx.FX_BH_FAST,
                                                  terms=True)
    finally:
        d.close()
    o = oracle.bh_forces(x, y, 0.5, 0.5, F32_01)
    assert np.array_equal(root, o["root"])
    assert np.array_equal(keys, o["keys"])
    assert np.array_equal(perm, o["perm"])
    assert np.array_equal(bx, o["fx32"]) and np.array_equal(by, o["fy32"])
    assert np.array_equal(bx, bx2) and np.array_equal(by, by2)
    num = np.sqrt(((bx - o["fx"]) ** 2 + (by - o["fy"]) ** 2).sum())
    assert num / np.sqrt((o["fx"] ** 2 + o["fy"] ** 2).sum()) < 1e-5
    # the hardware-rsqrt walk on the same (deep or shallow) tree
    assert np.array_equal(qkeys, keys) and np.array_equal(terms, o["interactions"])
    num = np.sqrt(((qx - o["fx"]) ** 2 + (qy - o["fy"]) ** 2).sum())
    assert num / np.sqrt((o["fx"] ** 2 + o["fy"] ** 2).sum()) < 1e-5
    return o


def test_deep_mode_on_a_large_die(fx, ctx, oracle):
    x, y = _crowded(4000.0)
    o = _check(fx, ctx, oracle, x, y, 4000.0)
    assert o["interactions"].max() < 400


def test_deep_kernels_launched_but_not_needed(fx, ctx, oracle):
    # a large die, but the points span ~600: the device keeps the 30-bit tree
    x, y = _crowded(600.0, seed=8)
    _check(fx, ctx, oracle, x, y, 4000.0)


def test_positions_outside_a_small_die(fx, ctx, oracle):
    # die 100, points over 3000: not in the die, so the device decides
    x, y = _crowded(3000.0, seed=9, clusters=5, per=800)
    _check(fx, ctx, oracle, x, y, 100.0)


def test_many_crowded_cells(fx, ctx, oracle):
    rng = np.random.default_rng(12)
    n = 120_000
    centers = rng.uniform(50, 2950, (300, 2))
    pts = (centers[rng.integers(0, 300, n)] + rng.uniform(0, 0.02, (n, 2))).astype(np.float32)
    _check(fx, ctx, oracle, pts[:, 0].copy(), pts[:, 1].copy(), 3000.0)


def test_fused_iterations_on_a_large_die(fx, ctx, oracle):
    """The plain iteration (attraction + Barnes-Hut + damped step) on a
    3000-wide die with crowded starting cells: the first iteration runs on
    uploaded positions, the next ones on clamped ones; the device run and the
    oracle's end on identical positions."""
    rng = np.random.default_rng(21)
    n = 6000
    nets = [list(rng.choice(n, size=rng.integers(2, 5), replace=False)) for _ in range(7000)]
    circ = fx.Circuit.from_nets(nets, n, 3000.0, 3000.0)
    centers = rng.uniform(100, 2900, (40, 2))
    p = (centers[rng.integers(0, 40, n)] + rng.uniform(0, 0.05, (n, 2))).astype(np.float32)
    x0, y0 = p[:, 0].copy(), p[:, 1].copy()
    cfg = fx.iter_cfg(density_bins=0, cong_cols=0, cong_rows=0, bh_walk=fx.FX_BH_EXACT)
    d = fx.Design(ctx, circ)
    try:
        x, y = x0.copy(), y0.copy()
        d.force_iterate(cfg, 10, x, y)  # eager, graph-replayed pairs, eager
    finally:
        d.close()
    rp, ri = oracle.build_adjacency(n, circ.net_ptr, circ.net_gate)
    ox, oy = x0.copy(), y0.copy()
    vx, vy = np.zeros_like(ox), np.zeros_like(oy)
    for _ in range(10):
        fa_x, fa_y = oracle.attraction_f32(rp, ri, ox, oy, 1.0)
        b = oracle.bh_forces(ox, oy, 0.5, 0.5, F32_01)
        oracle.integrate(ox, oy, vx, vy, fa_x + b["fx32"], fa_y + b["fy32"], 0.1, 0.9,
                         (0.0, 0.0, 3000.0, 3000.0))
    assert np.array_equal(x, ox) and np.array_equal(y, oy)

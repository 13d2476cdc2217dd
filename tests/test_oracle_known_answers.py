"""The CPU oracle against the reference's own unit-test known answers.

Each case ports an assertion of the reference's tests (file:line given).
"""
import numpy as np


def test_hpwl_square_is_20(oracle):
    # HAPR_fluxion_v4/src/data/placement.rs:87-96
    x = np.array([0, 10, 10, 0], np.float32)
    y = np.array([0, 0, 10, 10], np.float32)
    ptr, g = np.array([0, 4]), np.array([0, 1, 2, 3])
    assert abs(oracle.hpwl_f32(ptr, g, x, y) - 20.0) < 0.01
    assert oracle.hpwl_f64(ptr, g, x, y) == 20.0


def test_legacy_hpwl_30_and_wirelength_10(oracle):
    # neon_old_codebase/tests/python/test_benchmarks.py:249-265 (HPWL 30)
    x = np.array([0, 10], np.float32)
    y = np.array([0, 20], np.float32)
    assert oracle.hpwl_f64([0, 2], [0, 1], x, y) == 30.0
    # neon_old_codebase/tests/python/test_fluxion.py:178-186 (wirelength 10)
    assert oracle.hpwl_f64([0, 2], [0, 1], np.array([0, 10], np.float32),
                           np.zeros(2, np.float32)) == 10.0


def test_adjacency_known_answer(oracle):
    # HAPR_fluxion_v4/src/data/circuit.rs:200-216: nets {0,1}, {1,2}
    ap, ai = oracle.build_adjacency(3, [0, 2, 4], [0, 1, 1, 2])
    assert ai[ap[0]:ap[1]].tolist() == [1]
    assert ai[ap[1]:ap[2]].tolist() == [0, 2]
    assert ai[ap[2]:ap[3]].tolist() == [1]


def test_adjacency_dedup_and_self_pair(oracle):
    # circuit.rs:154-171: a pair shared by two nets appears once; a gate named
    # twice in one net lists itself once.
    ap, ai = oracle.build_adjacency(3, [0, 3, 5, 7], [0, 1, 2, 1, 0, 2, 2])
    assert ai[ap[0]:ap[1]].tolist() == [1, 2]
    assert ai[ap[1]:ap[2]].tolist() == [0, 2]
    assert ai[ap[2]:ap[3]].tolist() == [0, 1, 2]


def test_grid_cell_at_and_center(oracle):
    # HAPR_fluxion_v4/src/data/grid.rs:137-151
    cw, ch, cap = oracle.grid_geometry(100.0, 100.0, 10, 10)
    assert (oracle.cell_at(5.0, cw, 10), oracle.cell_at(5.0, ch, 10)) == (0, 0)
    assert (oracle.cell_at(95.0, cw, 10), oracle.cell_at(95.0, ch, 10)) == (9, 9)
    assert abs((0 + 0.5) * cw - 5.0) < 0.01
    h = np.zeros(100, np.float32)
    assert oracle.overflow(h, h, 10, 10, cap) == (0.0, 0.0)


def test_cell_at_saturating_cast(oracle):
    # Rust `as usize` saturates: negatives and NaN map to cell 0, huge values
    # to the last cell (grid.rs:58-62).
    assert oracle.cell_at(-5.0, 10.0, 10) == 0
    assert oracle.cell_at(float("nan"), 10.0, 10) == 0
    assert oracle.cell_at(1e30, 10.0, 10) == 9
    assert oracle.cell_at(float("inf"), 10.0, 10) == 9
    assert oracle.cell_at(100.0, 10.0, 10) == 9


def test_congestion_corner_net(oracle):
    # HAPR_fluxion_v4/src/algorithm/congestion.rs:100-117 (4 corner gates, one
    # net, 10 x 10 grid on 100 x 100): the box spans cells 1..9 both ways.
    x = np.array([10, 90, 10, 90], np.float32)
    y = np.array([10, 10, 90, 90], np.float32)
    h, v = oracle.congestion([0, 4], [0, 1, 2, 3], x, y, 100.0, 100.0, 10, 10)
    grid = h.reshape(10, 10)
    assert np.array_equal(h, v)
    assert grid[1:, 1:].sum() == 81 and grid.sum() == 81
    _, _, cap = oracle.grid_geometry(100.0, 100.0, 10, 10)
    tot, mx = oracle.overflow(h, v, 10, 10, cap)
    assert mx >= 0.0 and tot == 0.0


def test_hierarchy_two_leaves(oracle):
    # HAPR_fluxion_v4/src/data/hierarchy.rs:197-209: 6 gates in two leaves of
    # 3 -> depth 1, 3 nodes, 2 leaves.
    nets = [[i, i + 1] for i in range(5)]
    ptr = np.cumsum([0] + [2] * 5)
    ap, ai = oracle.build_adjacency(6, ptr, np.array(nets).ravel())
    h = oracle.build_hierarchy(6, ap, ai, 100.0, 100.0, max_leaf=3, min_cluster=1)
    assert h["max_depth"] == 1 and h["num_nodes"] == 3
    assert len(h["leaf_ptr"]) - 1 == 2


def test_partition_chain_covers_all(oracle):
    # HAPR_fluxion_v4/src/algorithm/partitioner.rs:232-251: a 20-gate chain
    # with max_leaf_size 8 covers all gates, depth >= 1, >= 2 leaves.
    nets = np.array([[i, i + 1] for i in range(19)]).ravel()
    ptr = np.arange(0, 39, 2)
    ap, ai = oracle.build_adjacency(20, ptr, nets)
    h = oracle.build_hierarchy(20, ap, ai, 1000.0, 1000.0, max_leaf=8)
    assert h["max_depth"] >= 1 and len(h["leaf_ptr"]) - 1 >= 2
    assert sorted(h["leaf_gate"].tolist()) == list(range(20))


def test_binary_regions_are_vertical_strips(oracle):
    # placer.rs:124-134: with two children, cols = ceil(sqrt 2) = 2 and
    # rows = 1, so every level halves the width only.
    nets = np.array([[i, i + 1] for i in range(15)]).ravel()
    ap, ai = oracle.build_adjacency(16, np.arange(0, 31, 2), nets)
    h = oracle.build_hierarchy(16, ap, ai, 100.0, 50.0, max_leaf=4)
    r = h["region"]
    assert np.all(r[:, 3] == 50.0)
    assert np.allclose(r[:, 2], 100.0 / 2 ** h["leaf_depth"])


def test_leaf_init_ignores_positions(oracle):
    # placer.rs:226-227: positions start at min + (i/n) w, (7i mod n)/n h; with
    # zero iterations the leaf is exactly that lattice.
    gates = np.arange(5)
    ap = np.zeros(6, np.int32)
    x, y = oracle.place_leaf(gates, ap, np.zeros(0, np.int32), (5.0, 5.0, 10.0, 10.0), 0)
    assert np.allclose(x, [0, 2, 4, 6, 8]) and np.allclose(y, [0, 4, 8, 2, 6])


def test_difference_array_congestion_matches_the_literal_loop(oracle):
    """oracle.congestion_counts (difference array, for full-size checks) gives
    the literal compute_congestion_cpu counts, edge cases included: pins
    outside the die, on its edges, negative, NaN, repeated, one-pin nets."""
    rng = np.random.default_rng(0)
    n, m = 3000, 2500
    x = rng.uniform(-5, 105, n).astype(np.float32)
    y = rng.uniform(-5, 85, n).astype(np.float32)
    x[:4] = [0.0, 100.0, np.nan, -0.0]
    y[:4] = [80.0, 0.0, 3.0, np.nan]
    deg = rng.integers(1, 9, m)
    ptr = np.concatenate([[0], np.cumsum(deg)]).astype(np.int32)
    gate = rng.integers(0, n, int(deg.sum())).astype(np.int32)
    gate[:8] = [0, 1, 2, 2, 3, 0, 1, 3]
    for cols, rows in [(64, 64), (37, 23), (1, 1)]:
        h, v = oracle.congestion(ptr, gate, x, y, 100.0, 80.0, cols, rows)
        c = oracle.congestion_counts(ptr, gate, x, y, 100.0, 80.0, cols, rows)
        assert np.array_equal(c.astype(np.float32), h) and np.array_equal(h, v)


def _place_gates_in_leaf_literal(gates, adjacency, region, iters, attract=1.0, repel=0.5,
                                 damping=0.9, dt=0.1):
    """placer.rs:210-287 line by line in numpy float32 scalars (every operation
    rounds to f32, as in Rust): the gate-to-slot map keeps a repeated gate's
    last slot (:232-235), springs go to the mapped slot (:243-255), and the
    final positions are written slot by slot (:283-286)."""
    f = np.float32
    cx, cy, w, h = (f(v) for v in region)
    n = len(gates)
    min_x, min_y = cx - w / f(2.0), cy - h / f(2.0)
    px = [min_x + (f(i) / f(n)) * w for i in range(n)]
    py = [min_y + (f(i * 7 % n) / f(n)) * h for i in range(n)]
    vx, vy = [f(0)] * n, [f(0)] * n
    g2l = {}
    for i, g in enumerate(gates):
        g2l[g] = i
    for _ in range(iters):
        fx, fy = [f(0)] * n, [f(0)] * n
        for g in gates:
            li = g2l[g]
            for nb in adjacency[g]:
                if nb in g2l:
                    lj = g2l[nb]
                    fx[li] = fx[li] + f(attract) * (px[lj] - px[li])
                    fy[li] = fy[li] + f(attract) * (py[lj] - py[li])
        for i in range(n):
            for j in range(i + 1, n):
                dx, dy = px[i] - px[j], py[i] - py[j]
                dist = max(np.sqrt(dx * dx + dy * dy), f(0.1))
                force = f(repel) / (dist * dist)
                fxij, fyij = force * dx / dist, force * dy / dist
                fx[i], fy[i] = fx[i] + fxij, fy[i] + fyij
                fx[j], fy[j] = fx[j] - fxij, fy[j] - fyij
        for i in range(n):
            vx[i] = (vx[i] + fx[i] * f(dt)) * f(damping)
            vy[i] = (vy[i] + fy[i] * f(dt)) * f(damping)
            px[i] = min(max(px[i] + vx[i] * f(dt), min_x), min_x + w)
            py[i] = min(max(py[i] + vy[i] * f(dt), min_y), min_y + h)
    out = {}
    for i, g in enumerate(gates):
        out[g] = (px[i], py[i])
    return out


def test_leaf_with_repeated_gates_matches_the_literal_loop(oracle):
    """A leaf listing gates 3 and 1 twice: the oracle's place_leaf gives the
    literal loop's positions bit for bit (springs on the last slot, last slot
    written)."""
    adjacency = {0: [1], 1: [0, 2, 3], 2: [1, 3], 3: [1, 2, 4], 4: [3]}
    ap = np.zeros(6, np.int32)
    ai = []
    for g in range(5):
        ai += adjacency[g]
        ap[g + 1] = len(ai)
    gates = [3, 1, 3, 2, 1, 4]
    region = (2.0, 3.0, 4.0, 2.0)
    want = _place_gates_in_leaf_literal(gates, adjacency, region, 12)
    x = np.full(5, 9.0, np.float32)
    y = np.full(5, 9.0, np.float32)
    oracle.place_leaf(np.array(gates), ap, np.array(ai, np.int32), region, 12, 1.0, 0.5, 0.9,
                      0.1, x, y)
    for g, (wx, wy) in want.items():
        assert x[g] == wx and y[g] == wy, g
    assert x[0] == 9.0 and y[0] == 9.0  # not in the leaf

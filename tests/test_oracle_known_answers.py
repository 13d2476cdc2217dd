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


def _sinf():
    """The platform C library's sinf, which Rust's f32::sin calls on Linux."""
    import ctypes
    import ctypes.util
    libm = ctypes.CDLL(ctypes.util.find_library("m"))
    libm.sinf.restype = ctypes.c_float
    libm.sinf.argtypes = [ctypes.c_float]
    return lambda v: np.float32(libm.sinf(float(v)))


def _fiedler_literal(gates, adjacency, iters):
    """partitioner.rs:106-185 compute_fiedler_vector line by line in float32."""
    f = np.float32
    sinf = _sinf()
    n = len(gates)
    if n <= 1:
        return [f(0)] * n
    g2l = {}
    for i, g in enumerate(gates):
        g2l[g] = i
    degree = [f(0)] * n
    pairs = []
    for g in gates:
        for nb in adjacency[g]:
            if nb in g2l:
                lg = g2l[g]
                pairs.append((lg, g2l[nb]))
                degree[lg] = degree[lg] + f(1.0)
    v = [sinf(f(i) * f(2.71828)) for i in range(n)]
    norm = f(0)
    for t in v:
        norm = norm + t * t
    norm = np.sqrt(norm)
    if norm > f(1e-10):
        v = [t / norm for t in v]
    for _ in range(iters):
        lv = [degree[i] * v[i] for i in range(n)]
        for i, j in pairs:
            lv[i] = lv[i] - v[j]
        s = f(0)
        for t in lv:
            s = s + t
        mean = s / f(n)
        lv = [t - mean for t in lv]
        norm = f(0)
        for t in lv:
            norm = norm + t * t
        norm = np.sqrt(norm)
        if norm > f(1e-10):
            lv = [t / norm for t in lv]
        v = lv
    return v


def test_fiedler_matches_the_literal_loop(oracle):
    """The oracle's compute_fiedler_vector against a literal float32
    transcription on a 40-gate subset of a random netlist (subset listed out
    of order), 30 iterations: every component bit for bit."""
    rng = np.random.default_rng(4)
    n = 60
    nets = [list(rng.choice(n, size=rng.integers(2, 5), replace=False)) for _ in range(90)]
    ptr = np.zeros(len(nets) + 1, np.int32)
    for e, net in enumerate(nets):
        ptr[e + 1] = ptr[e] + len(net)
    ap, ai = oracle.build_adjacency(n, ptr, np.concatenate(nets).astype(np.int32))
    adjacency = {g: list(ai[ap[g]:ap[g + 1]]) for g in range(n)}
    gates = [int(g) for g in rng.permutation(n)[:40]]
    want = _fiedler_literal(gates, adjacency, 30)
    got = oracle.fiedler_vector(ap, ai, np.array(gates), 30)
    assert np.array_equal(got, np.array(want, np.float32))


def _refine_literal(net_ptr, net_gate, x, y, chip_w, chip_h, max_iters, max_move, threshold,
                    cols, rows):
    """refiner.rs:34-126 with grid.rs and congestion.rs:11-93, line by line in
    float32; returns the positions and the number of iterations that moved
    gates."""
    f = np.float32
    x, y = [f(v) for v in x], [f(v) for v in y]
    cw, ch = f(chip_w) / f(cols), f(chip_h) / f(rows)
    cap = (cw + ch) * f(0.5)

    def cell_at(px, py):
        def cast(v):  # Rust's saturating `as usize`
            return 0 if not v > 0 else int(min(float(v), 2.0 ** 64 - 1))
        return min(cast(px / cw), cols - 1), min(cast(py / ch), rows - 1)

    def congestion():
        h = [f(0)] * (cols * rows)
        for e in range(len(net_ptr) - 1):
            gs = net_gate[net_ptr[e]:net_ptr[e + 1]]
            if len(gs) < 2:
                continue
            mnx, mxx = f(np.finfo(np.float32).max), f(np.finfo(np.float32).min)
            mny, mxy = mnx, mxx
            for g in gs:
                mnx, mxx = min(mnx, x[g]), max(mxx, x[g])
                mny, mxy = min(mny, y[g]), max(mxy, y[g])
            c0, r0 = cell_at(mnx, mny)
            c1, r1 = cell_at(mxx, mxy)
            for r in range(r0, r1 + 1):
                for c in range(c0, c1 + 1):
                    h[r * cols + c] = h[r * cols + c] + f(1.0)
        return h  # v equals h cell for cell

    def overflow(h, c, r):
        t = h[r * cols + c] + h[r * cols + c]
        return max(t - cap, f(0.0))

    prev, stall, moved_iters = f(np.finfo(np.float32).max), 0, 0
    for _ in range(max_iters):
        h = congestion()
        total = f(0)
        for r in range(rows):
            for c in range(cols):
                total = total + overflow(h, c, r)
        if total <= f(threshold):
            break
        if abs(prev - total) < f(0.01) * max(prev, f(1.0)):
            stall += 1
            if stall >= 10:
                break
        else:
            stall = 0
        prev = total
        hot = {(c, r) for r in range(rows) for c in range(cols)
               if overflow(h, c, r) > f(threshold)}
        for g in [g for g in range(len(x)) if cell_at(x[g], y[g]) in hot]:
            gx, gy = x[g], y[g]
            col, row = cell_at(gx, gy)
            best = None
            for dr in range(-3, 4):
                for dc in range(-3, 4):
                    if dr == 0 and dc == 0:
                        continue
                    nc, nr = col + dc, row + dr
                    if 0 <= nc < cols and 0 <= nr < rows:
                        t = h[nr * cols + nc] + h[nr * cols + nc]
                        if best is None or t < best[0]:
                            best = (t, nc, nr)
            if best is None:
                continue
            tx, ty = (f(best[1]) + f(0.5)) * cw, (f(best[2]) + f(0.5)) * ch
            dx = min(max(tx - gx, f(-max_move)), f(max_move))
            dy = min(max(ty - gy, f(-max_move)), f(max_move))
            x[g] = min(max(gx + dx, f(0.0)), f(chip_w))
            y[g] = min(max(gy + dy, f(0.0)), f(chip_h))
        moved_iters += 1
    return np.array(x, np.float32), np.array(y, np.float32), moved_iters


def test_refine_matches_the_literal_loop(oracle):
    """The oracle's refine_placement against a literal float32 transcription:
    80 gates crowded into one corner of a 40 x 40 die, 8 x 8 grid, up to 25
    iterations; positions bit for bit and the same number of moving iterations."""
    rng = np.random.default_rng(8)
    n = 80
    nets = [list(rng.choice(n, size=rng.integers(2, 4), replace=False)) for _ in range(120)]
    ptr = np.zeros(len(nets) + 1, np.int32)
    for e, net in enumerate(nets):
        ptr[e + 1] = ptr[e] + len(net)
    gate = np.concatenate(nets).astype(np.int32)
    x0 = rng.uniform(0, 12, n).astype(np.float32)
    y0 = rng.uniform(0, 12, n).astype(np.float32)
    wx, wy, wit = _refine_literal(ptr, gate, x0, y0, 40.0, 40.0, 25, 5.0, 1.0, 8, 8)
    gx, gy, git, _ = oracle.refine(ptr, gate, x0, y0, 40.0, 40.0, max_iters=25,
                                   move_distance=5.0, threshold=1.0, cols=8, rows=8)
    assert wit > 0
    assert np.array_equal(gx, wx) and np.array_equal(gy, wy) and git == wit


def test_attraction_and_damped_step_match_the_literal_loops(oracle):
    """The plain iteration's spring forces (placer.rs:243-255 over every gate:
    F_g += k (p_nb - p_g) in adjacency order) and damped step
    (placer.rs:275-280 with Rust's clamp to the die) against literal float32
    loops, bit for bit."""
    f = np.float32
    rng = np.random.default_rng(6)
    n = 50
    nets = [list(rng.choice(n, size=rng.integers(2, 6), replace=False)) for _ in range(70)]
    ptr = np.zeros(len(nets) + 1, np.int32)
    for e, net in enumerate(nets):
        ptr[e + 1] = ptr[e] + len(net)
    ap, ai = oracle.build_adjacency(n, ptr, np.concatenate(nets).astype(np.int32))
    x = rng.uniform(0, 30, n).astype(np.float32)
    y = rng.uniform(0, 30, n).astype(np.float32)
    k = 0.75
    fx, fy = oracle.attraction_f32(ap, ai, x, y, k)
    for g in range(n):
        ax = ay = f(0)
        for q in range(ap[g], ap[g + 1]):
            ax = ax + f(k) * (x[ai[q]] - x[g])
            ay = ay + f(k) * (y[ai[q]] - y[g])
        assert fx[g] == ax and fy[g] == ay, g
    vx = rng.normal(0, 3, n).astype(np.float32)
    vy = rng.normal(0, 3, n).astype(np.float32)
    forces_x = (fx * f(40)).astype(np.float32)  # large enough to push some gates off the die
    forces_y = (fy * f(40)).astype(np.float32)
    ox, oy, ovx, ovy = x.copy(), y.copy(), vx.copy(), vy.copy()
    oracle.integrate(ox, oy, ovx, ovy, forces_x, forces_y, 0.1, 0.9, (0.0, 0.0, 30.0, 30.0))
    clamped = 0
    for g in range(n):
        wvx = (vx[g] + forces_x[g] * f(0.1)) * f(0.9)
        wvy = (vy[g] + forces_y[g] * f(0.1)) * f(0.9)
        px, py = x[g] + wvx * f(0.1), y[g] + wvy * f(0.1)
        wx = min(max(px, f(0.0)), f(30.0))
        wy = min(max(py, f(0.0)), f(30.0))
        clamped += (wx != px) + (wy != py)
        assert (ovx[g], ovy[g], ox[g], oy[g]) == (wvx, wvy, wx, wy), g
    assert clamped > 0


def _bisect_literal(gates, adjacency, depth, leaves, counter, max_leaf=64, min_cluster=8,
                    balance=0.4, iters=30):
    """partitioner.rs:63-104 recursive_bisect and :186-212 split_by_fiedler
    line by line (Rust's sort_by is stable, as is Python's sort)."""
    counter[0] += 1
    n = len(gates)
    if n <= max_leaf or n <= min_cluster:
        leaves.append((list(gates), depth))
        return
    fiedler = _fiedler_literal(gates, adjacency, iters)
    order = sorted(range(n), key=lambda i: fiedler[i])
    min_size = int(np.ceil(np.float32(n) * np.float32(balance)))
    split = min(max(n // 2, min_size), n - min_size)
    left = [gates[i] for i in order[:split]]
    right = [gates[i] for i in order[split:]]
    if not left or not right:
        leaves.append((list(gates), depth))
        return
    _bisect_literal(left, adjacency, depth + 1, leaves, counter, max_leaf, min_cluster, balance,
                    iters)
    _bisect_literal(right, adjacency, depth + 1, leaves, counter, max_leaf, min_cluster, balance,
                    iters)


def test_hierarchy_matches_the_literal_bisection(oracle):
    """The oracle's build_hierarchy against a literal recursive_bisect over the
    literal Fiedler vector: 400 gates of a random netlist, default partition
    settings; the same leaves (gates in order), depths and node count."""
    rng = np.random.default_rng(10)
    n = 400
    nets = [list(rng.choice(n, size=rng.integers(2, 5), replace=False)) for _ in range(520)]
    ptr = np.zeros(len(nets) + 1, np.int32)
    for e, net in enumerate(nets):
        ptr[e + 1] = ptr[e] + len(net)
    ap, ai = oracle.build_adjacency(n, ptr, np.concatenate(nets).astype(np.int32))
    adjacency = {g: list(ai[ap[g]:ap[g + 1]]) for g in range(n)}
    leaves, counter = [], [0]
    _bisect_literal(list(range(n)), adjacency, 0, leaves, counter)
    h = oracle.build_hierarchy(n, ap, ai, 100.0, 100.0)
    lp, lg = h["leaf_ptr"], h["leaf_gate"]
    assert len(leaves) > 4 and len(lp) - 1 == len(leaves)
    for l, (gs, depth) in enumerate(leaves):
        assert list(lg[lp[l]:lp[l + 1]]) == gs and h["leaf_depth"][l] == depth, l
    assert h["num_nodes"] == counter[0]


def test_circuit_basic_shared_and_touching_counts(oracle):
    # circuit.rs:196-217 test_circuit_basic: nets {0,1}, {1,2};
    # count_shared_nets([0], [1]) = 1 and count_nets_touching([1]) = 2. In the
    # attention score shared / touching(i) (attention.rs:64-72) that is
    # scores[1][0] = 1 / 2 and scores[0][1] = 1 / 1; gates 0 and 2 share none.
    scores, tops = oracle.attention_level([0, 2, 4], [0, 1, 1, 2], [[0], [1], [2]], top_k=10)
    want = np.array([[0, 1, 0], [0.5, 0, 0.5], [0, 1, 0]], np.float32)
    assert np.array_equal(scores, want)
    assert tops == [[1], [0, 2], [1]]


def test_composite_iteration_oracle_is_consistent(oracle):
    """plain_forces (the checker of the benchmarked step): its f32 sum agrees
    with its FP64 recomputation to f32 rounding, the density term is the
    FP64 density_forces of the same positions, and plain_run's first step is
    the damped step of those f32 forces."""
    rng = np.random.default_rng(3)
    n, die = 3000, 60.0
    nets = [rng.choice(n, size=rng.integers(2, 6), replace=False) for _ in range(3600)]
    net_ptr = np.concatenate([[0], np.cumsum([len(e) for e in nets])]).astype(np.int32)
    net_gate = np.concatenate(nets).astype(np.int32)
    ap, ai = oracle.build_adjacency(n, net_ptr, net_gate)
    x = rng.uniform(0, die, n).astype(np.float32)
    y = rng.uniform(0, die, n).astype(np.float32)
    area = rng.integers(1, 5, n).astype(np.float32)
    md = float(np.float32(0.1))
    base = oracle.plain_forces(ap, ai, x, y, area, die, die, min_dist=md)
    full = oracle.plain_forces(ap, ai, x, y, area, die, die, min_dist=md, bins=64, weight=1.0)
    d = oracle.density_forces(x, y, area.astype(np.float64), die, die, 64, 0.7, 1.0)
    assert np.allclose(full["f64"][0] - base["f64"][0], d["fx"], rtol=1e-12, atol=1e-9)
    assert np.allclose(full["f64"][1] - base["f64"][1], d["fy"], rtol=1e-12, atol=1e-9)
    for r in (base, full):
        num = np.sqrt(sum(((a.astype(np.float64) - b) ** 2).sum() for a, b in zip(r["f32"], r["f64"])))
        den = np.sqrt(sum((b ** 2).sum() for b in r["f64"]))
        assert num <= 1e-6 * den
    rx, ry = oracle.plain_run(ap, ai, x, y, area, die, die, 1, min_dist=md, bins=64, weight=1.0)
    ox, oy = x.copy(), y.copy()
    vx, vy = np.zeros_like(ox), np.zeros_like(oy)
    oracle.integrate(ox, oy, vx, vy, *full["f32"], 0.1, 0.9, (0.0, 0.0, die, die))
    assert np.array_equal(rx, ox) and np.array_equal(ry, oy)

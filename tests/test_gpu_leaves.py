"""Row H: the batched leaf placer against the oracle's literal restatement of
place_gates_in_leaf (HAPR_fluxion_v4/src/algorithm/placer.rs:210-287)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_leaves(oracle, s, iters):
    c = s.circuit
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    ox = np.zeros(c.num_gates, np.float32)
    oy = np.zeros(c.num_gates, np.float32)
    lp, reg = s.leaf_ptr, s.region.reshape(-1, 4)
    gates = np.arange(c.num_gates, dtype=np.int32)
    for l in range(len(lp) - 1):
        oracle.place_leaf(gates[lp[l]:lp[l + 1]], ap, ai, reg[l], iters, 1.0, 0.5, 0.9, 0.1,
                          ox, oy)
    return ox, oy


@pytest.fixture(scope="module")
def batch(fx):
    return fx.synth_leaves(7, 192, 16, 128, 1.5)


SCHEDULES = ["warp", "cta64", "cta128", "cta256", "pair64", "pair128", "pair256",
             "per_cluster"]


def _code(fx, schedule):
    return {"warp": fx.FX_LEAF_WARP, "cta64": fx.FX_LEAF_CTA64, "cta128": fx.FX_LEAF_CTA128,
            "cta256": fx.FX_LEAF_CTA256, "pair64": fx.FX_LEAF_PAIR64,
            "pair128": fx.FX_LEAF_PAIR128, "pair256": fx.FX_LEAF_PAIR256,
            "per_cluster": fx.FX_LEAF_PER_CLUSTER}[schedule]


@pytest.mark.parametrize("schedule", SCHEDULES)
def test_leaf_schedules_bit_exact(fx, ctx, oracle, batch, schedule):
    code = _code(fx, schedule)
    d = fx.Design(ctx, batch.circuit)
    try:
        cfg = fx.leaf_cfg(force_iterations=60, schedule=code)
        gates = np.arange(batch.circuit.num_gates, dtype=np.int32)
        x, y, used = d.place_leaves(batch.leaf_ptr, gates, batch.region, cfg)
    finally:
        d.close()
    assert used == code
    ox, oy = _oracle_leaves(oracle, batch, 60)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)


def test_leaf_autotune_and_full_run(fx, ctx, oracle):
    """300 iterations (the batched-leaf workload's count) on 48 clusters,
    autotuned schedule: bit-identical to the reference loop."""
    s = fx.synth_leaves(11, 48, 16, 128, 1.5)
    d = fx.Design(ctx, s.circuit)
    try:
        gates = np.arange(s.circuit.num_gates, dtype=np.int32)
        x, y, used = d.place_leaves(s.leaf_ptr, gates, s.region,
                                    fx.leaf_cfg(force_iterations=300))
    finally:
        d.close()
    assert used in (fx.FX_LEAF_WARP, fx.FX_LEAF_CTA64, fx.FX_LEAF_CTA128, fx.FX_LEAF_CTA256,
                    fx.FX_LEAF_PAIR64, fx.FX_LEAF_PAIR128, fx.FX_LEAF_PAIR256)
    ox, oy = _oracle_leaves(oracle, s, 300)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)


def test_leaf_regions_and_untouched_gates(fx, ctx, oracle):
    """Leaves on distinct regions (the hierarchy's vertical strips), a leaf of
    one gate, an empty leaf, and gates outside every leaf keeping their input
    positions."""
    s = fx.synth_plain(4, 600, 700, 40.0)
    c = s.circuit
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    h = oracle.build_hierarchy(c.num_gates, ap, ai, c.chip_width, c.chip_height)
    lp, lg, reg = h["leaf_ptr"].copy(), h["leaf_gate"].copy(), h["region"].copy()
    # drop the last leaf's gates from the batch and add a 1-gate and an empty leaf
    keep = lp[-2]
    dropped = lg[keep:].copy()
    lg2 = np.concatenate([lg[:keep], dropped[:1]])
    lp2 = np.concatenate([lp[:-1], [keep + 1, keep + 1]]).astype(np.int32)
    reg2 = np.concatenate([reg[:-1], reg[-1:], reg[-1:]])
    x0 = np.full(c.num_gates, 7.0, np.float32)
    d = fx.Design(ctx, c)
    try:
        x, y, _ = d.place_leaves(lp2, lg2, reg2, fx.leaf_cfg(force_iterations=50),
                                 x0, x0.copy())
    finally:
        d.close()
    ox, oy = x0.copy(), x0.copy()
    for l in range(len(lp2) - 1):
        oracle.place_leaf(lg2[lp2[l]:lp2[l + 1]], ap, ai, reg2[l], 50, 1.0, 0.5, 0.9, 0.1,
                          ox, oy)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)
    assert np.all(x[dropped[1:]] == 7.0)


def test_leaf_too_large_is_rejected(fx, ctx):
    s = fx.synth_plain(4, 600, 700, 40.0)
    d = fx.Design(ctx, s.circuit)
    try:
        with pytest.raises(fx.FluxionError):
            d.place_leaves([0, 600], np.arange(600), [20, 20, 40, 40])
    finally:
        d.close()


def _every_size_batch(fx, sizes, seed):
    """One leaf of each listed size, gates numbered leaf by leaf, nets of 2-4
    pins inside each leaf, every leaf on its own unit box."""
    rng = np.random.default_rng(seed)
    nets, base = [], 0
    for n in sizes:
        for _ in range(int(1.5 * n) if n > 1 else 0):
            k = min(n, int(rng.integers(2, 5)))
            nets.append(list(base + rng.choice(n, size=k, replace=False)))
        base += n
    if not nets:
        nets = [[0, 0]]
    circ = fx.Circuit.from_nets(nets, base, float(len(sizes)), 1.0)
    lp = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    reg = np.array([[l + 0.5, 0.5, 1.0, 1.0] for l in range(len(sizes))], np.float32)
    return circ, lp, reg


@pytest.mark.parametrize("schedule", ["pair64", "pair128", "pair256", "cta64"])
def test_leaf_every_size_up_to_128(fx, ctx, oracle, schedule):
    """Leaves of 1..128 gates (both parities of n, a leaf of one gate, the
    128-gate maximum of the pair schedules), shuffled: every schedule lands on
    the reference's positions bit for bit."""
    sizes = np.random.default_rng(3).permutation(np.arange(1, 129))
    circ, lp, reg = _every_size_batch(fx, sizes, 5)
    gates = np.arange(circ.num_gates, dtype=np.int32)
    d = fx.Design(ctx, circ)
    try:
        x, y, used = d.place_leaves(lp, gates, reg.ravel(),
                                    fx.leaf_cfg(force_iterations=25, schedule=_code(fx, schedule)))
    finally:
        d.close()
    assert used == _code(fx, schedule)
    ap, ai = oracle.build_adjacency(circ.num_gates, circ.net_ptr, circ.net_gate)
    ox = np.zeros(circ.num_gates, np.float32)
    oy = np.zeros(circ.num_gates, np.float32)
    for l in range(len(sizes)):
        oracle.place_leaf(gates[lp[l]:lp[l + 1]], ap, ai, reg[l], 25, 1.0, 0.5, 0.9, 0.1,
                          ox, oy)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)


def test_leaf_pair_schedules_take_at_most_128_gates(fx, ctx, oracle):
    """A batch with a 129-gate leaf: the pair schedules refuse it, and the
    autotuner picks among the others (the result still matches)."""
    sizes = np.array([129, 40, 7])
    circ, lp, reg = _every_size_batch(fx, sizes, 9)
    gates = np.arange(circ.num_gates, dtype=np.int32)
    d = fx.Design(ctx, circ)
    try:
        with pytest.raises(fx.FluxionError):
            d.place_leaves(lp, gates, reg.ravel(),
                           fx.leaf_cfg(force_iterations=5, schedule=fx.FX_LEAF_PAIR128))
        x, y, used = d.place_leaves(lp, gates, reg.ravel(), fx.leaf_cfg(force_iterations=5))
    finally:
        d.close()
    assert used in (fx.FX_LEAF_WARP, fx.FX_LEAF_CTA64, fx.FX_LEAF_CTA128, fx.FX_LEAF_CTA256)
    ap, ai = oracle.build_adjacency(circ.num_gates, circ.net_ptr, circ.net_gate)
    ox = np.zeros(circ.num_gates, np.float32)
    oy = np.zeros(circ.num_gates, np.float32)
    for l in range(len(sizes)):
        oracle.place_leaf(gates[lp[l]:lp[l + 1]], ap, ai, reg[l], 5, 1.0, 0.5, 0.9, 0.1,
                          ox, oy)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)


@pytest.mark.parametrize("sizes,iters", [
    ([90, 64, 63, 62, 40, 17, 2, 1], 30),   # largest 90: halves take leaves <= 62
    ([2, 1, 2, 1, 1], 12),                  # largest 2: one-gate leaves run two to a block
    ([128, 91, 90, 3], 0),                  # no iterations: the initial layout
    ([128, 91, 90, 3], 1),
])
@pytest.mark.parametrize("schedule", ["pair64", "pair128", "pair256"])
def test_leaf_pair_split_points(fx, ctx, oracle, schedule, sizes, iters):
    """The pair schedules hand the largest leaves to whole blocks and the rest
    to half blocks, by a split the host derives from the largest leaf: batches
    whose largest leaf sits at, above and below the split, leaves of one and
    two gates, and zero or one iteration, against the reference loop."""
    sizes = np.array(sizes)
    circ, lp, reg = _every_size_batch(fx, sizes, 13)
    gates = np.arange(circ.num_gates, dtype=np.int32)
    d = fx.Design(ctx, circ)
    try:
        x, y, _ = d.place_leaves(lp, gates, reg.ravel(),
                                 fx.leaf_cfg(force_iterations=iters, schedule=_code(fx, schedule)))
    finally:
        d.close()
    ap, ai = oracle.build_adjacency(circ.num_gates, circ.net_ptr, circ.net_gate)
    ox = np.zeros(circ.num_gates, np.float32)
    oy = np.zeros(circ.num_gates, np.float32)
    for l in range(len(sizes)):
        oracle.place_leaf(gates[lp[l]:lp[l + 1]], ap, ai, reg[l], iters, 1.0, 0.5, 0.9, 0.1,
                          ox, oy)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)


@pytest.mark.parametrize("schedule", ["warp", "cta64", "pair128", "pair256", "per_cluster"])
def test_leaf_repeated_gates_keep_the_last_slot(fx, ctx, oracle, schedule):
    """A gate listed twice in one leaf, and a gate listed in two leaves: the
    reference writes positions slot by slot, leaf by leaf, so the last listing
    wins; a gate that lost its only slot to a repeat keeps its input position."""
    sizes = np.array([20, 30, 25, 40])
    circ, lp, reg = _every_size_batch(fx, sizes, 21)
    lg = np.arange(circ.num_gates, dtype=np.int32)
    lg[5] = lg[2]                 # within leaf 0
    lg[lp[2]] = lg[lp[1] + 7]     # leaf 2 repeats a gate of leaf 1
    lg[lp[3] + 39] = lg[lp[3]]    # within leaf 3, the last slot repeats the first
    x0 = np.full(circ.num_gates, 3.25, np.float32)
    d = fx.Design(ctx, circ)
    try:
        x, y, _ = d.place_leaves(lp, lg, reg.ravel(),
                                 fx.leaf_cfg(force_iterations=20, schedule=_code(fx, schedule)),
                                 x0, x0.copy())
    finally:
        d.close()
    ap, ai = oracle.build_adjacency(circ.num_gates, circ.net_ptr, circ.net_gate)
    ox, oy = x0.copy(), x0.copy()
    for l in range(len(sizes)):
        oracle.place_leaf(lg[lp[l]:lp[l + 1]], ap, ai, reg[l], 20, 1.0, 0.5, 0.9, 0.1, ox, oy)
    assert np.array_equal(x, ox) and np.array_equal(y, oy)
    assert x[5] == 3.25 and x[lp[2]] == 3.25  # their slots went to repeats

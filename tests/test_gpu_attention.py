"""(f.4) attention scores (compute_level_attention,
HAPR_fluxion_v4/src/algorithm/attention.rs:50-88) on the device against the
oracle: scores bit-exact (integer counts, one f32 division) and identical
top-k lists."""
import numpy as np
import pytest

from test_attention_host import _random_level

pytestmark = pytest.mark.gpu


def _design(fx, ctx, n_gates, net_ptr, net_gate):
    c = fx.Circuit(n_gates, np.asarray(net_ptr, np.int32), np.asarray(net_gate, np.int32),
                   np.full(n_gates, 2.0, np.float32), np.full(n_gates, 10.0, np.float32),
                   100.0, 100.0, "attention", None)
    return fx.Design(ctx, c)


@pytest.mark.parametrize("seed,top_k", [(0, 10), (1, 1), (2, 0), (3, 64)])
def test_level_matches_the_literal_oracle(fx, ctx, oracle, seed, top_k):
    rng = np.random.default_rng(seed)
    n_gates, n_clusters = 400, 37
    net_ptr, net_gate, cp, cg = _random_level(rng, n_gates, 350, n_clusters)
    net_gate[1] = net_gate[0]  # a gate named twice in one net
    d = _design(fx, ctx, n_gates, net_ptr, net_gate)
    try:
        top, sc = d.attention_level(cp, cg, top_k, scores=True)
    finally:
        d.close()
    clusters = [cg[cp[i]:cp[i + 1]].tolist() for i in range(n_clusters)]
    s, want = oracle.attention_level(net_ptr, net_gate, clusters, top_k)
    assert np.array_equal(sc.view(np.uint32), s.view(np.uint32))
    assert [[j for j in r if j >= 0] for r in top.tolist()] == want
    assert top.shape == (n_clusters, top_k)


def test_large_level_matches_the_sparse_oracle(fx, ctx, oracle):
    rng = np.random.default_rng(11)
    n_gates, n_clusters = 200_000, 6000
    net_ptr, net_gate, cp, cg = _random_level(rng, n_gates, 240_000, n_clusters, max_pins=12,
                                              outside=0.02)
    d = _design(fx, ctx, n_gates, net_ptr, net_gate)
    try:
        top, _ = d.attention_level(cp, cg, 10)
        top2, _ = d.attention_level(cp, cg, 10)
    finally:
        d.close()
    _, _, _, want = oracle.attention_level_sparse(net_ptr, net_gate, n_gates, cp, cg, 10)
    assert np.array_equal(top, want)
    assert np.array_equal(top, top2)


def test_all_levels_of_a_device_hierarchy(fx, ctx, oracle, plain_small):
    c = plain_small.circuit
    d = fx.Design(ctx, c)
    try:
        tree = d.partition(fx.part_cfg())
        levels = d.attention(tree, top_k=10, scores=True)
    finally:
        d.close()
    ref = fx.hierarchy_levels(tree["leaf_ptr"], tree["leaf_gate"], tree["leaf_depth"])
    want_depths = [t for t, (cp, _) in enumerate(ref) if len(cp) - 1 >= 2]
    assert [lv["level_index"] for lv in levels] == want_depths and want_depths[0] == 1
    for lv in levels:
        cp, cg = ref[lv["level_index"]]
        r, col, v, tk = oracle.attention_level_sparse(c.net_ptr, c.net_gate, c.num_gates,
                                                      cp, cg, 10)
        dense = np.zeros_like(lv["scores"])
        dense[r, col] = v
        assert np.array_equal(lv["scores"].view(np.uint32), dense.view(np.uint32))
        assert fx.top_k_lists(lv["top_k"]) == fx.top_k_lists(tk)


def test_edge_cases(fx, ctx, oracle):
    net_ptr = np.array([0, 2, 4, 6], np.int32)
    net_gate = np.array([0, 1, 0, 3, 3, 4], np.int32)
    d = _design(fx, ctx, 6, net_ptr, net_gate)
    try:
        # the reference's unit test (attention.rs:107-126)
        top, sc = d.attention_level([0, 3, 6], [0, 1, 2, 3, 4, 5], 5, scores=True)
        assert sc.tolist() == [[0.0, 0.5], [0.5, 0.0]]
        assert top.tolist() == [[1, -1, -1, -1, -1], [0, -1, -1, -1, -1]]
        # no clusters; one cluster; a cluster touching no net
        assert d.attention_level([0], [], 3, scores=True)[0].shape == (0, 3)
        top, sc = d.attention_level([0, 6], [0, 1, 2, 3, 4, 5], 3, scores=True)
        assert top.tolist() == [[-1, -1, -1]] and sc.tolist() == [[0.0]]
        top, sc = d.attention_level([0, 1, 2], [5, 2], 3, scores=True)
        assert np.all(top == -1) and np.all(sc == 0)
        # malformed levels are refused
        with pytest.raises(fx.FluxionError):
            d.attention_level([0, 2, 4], [0, 1, 1, 2], 3)  # gate 1 in two clusters
        with pytest.raises(fx.FluxionError):
            d.attention_level([0, 2], [0, 9], 3)  # gate out of range
        with pytest.raises(fx.FluxionError):
            d.attention_level([0, 2, 1], [0, 1], 3)  # decreasing cluster_ptr
    finally:
        d.close()


def test_high_fanout_nets(fx, ctx, oracle):
    """Nets beyond one warp's 32 pins take the block path (a bitmap of the
    level's clusters): degrees 33..600, repeated gates, pins outside every
    cluster, and one net over almost all gates."""
    rng = np.random.default_rng(17)
    n_gates, n_clusters = 700, 61
    degs = np.concatenate([rng.integers(2, 9, 150), [33, 40, 64, 65, 127, 300, 600, 690]])
    rng.shuffle(degs)
    net_ptr = np.concatenate([[0], np.cumsum(degs)]).astype(np.int32)
    net_gate = rng.integers(0, n_gates, int(degs.sum())).astype(np.int32)
    gates = rng.permutation(n_gates)[:650].astype(np.int32)
    cuts = np.sort(rng.choice(np.arange(1, 650), n_clusters - 1, replace=False))
    cp = np.concatenate([[0], cuts, [650]]).astype(np.int32)
    d = _design(fx, ctx, n_gates, net_ptr, net_gate)
    try:
        top, sc = d.attention_level(cp, gates, 12, scores=True)
        top2, sc2 = d.attention_level(cp, gates, 12, scores=True)
    finally:
        d.close()
    clusters = [gates[cp[i]:cp[i + 1]].tolist() for i in range(n_clusters)]
    s, want = oracle.attention_level(net_ptr, net_gate, clusters, 12)
    assert np.array_equal(sc.view(np.uint32), s.view(np.uint32))
    assert [[j for j in r if j >= 0] for r in top.tolist()] == want
    assert np.array_equal(top, top2) and np.array_equal(sc, sc2)


@pytest.mark.parametrize("n_clusters,top_k", [(100, 10), (5000, 10), (5000, 40), (20_000, 10)])
def test_many_clusters_with_big_nets(fx, ctx, oracle, n_clusters, top_k):
    """The three count paths: an n x n matrix per block (n <= 128), a block
    per row (n <= 16384) and the pair hash table beyond; top-10 and, through
    the block-per-row path, top-40 lists."""
    rng = np.random.default_rng(23)
    n_gates = 120_000
    degs = np.where(rng.random(90_000) < 0.01, rng.integers(33, 200, 90_000),
                    rng.integers(2, 8, 90_000))
    net_ptr = np.concatenate([[0], np.cumsum(degs)]).astype(np.int32)
    net_gate = rng.integers(0, n_gates, int(degs.sum())).astype(np.int32)
    gates = rng.permutation(n_gates).astype(np.int32)
    cuts = np.sort(rng.choice(np.arange(1, n_gates), n_clusters - 1, replace=False))
    cp = np.concatenate([[0], cuts, [n_gates]]).astype(np.int32)
    d = _design(fx, ctx, n_gates, net_ptr, net_gate)
    try:
        top, _ = d.attention_level(cp, gates, top_k)
    finally:
        d.close()
    _, _, _, want = oracle.attention_level_sparse(net_ptr, net_gate, n_gates, cp, gates, top_k)
    assert np.array_equal(top, want)


def test_whole_hierarchy_call_matches_the_levels(fx, ctx, oracle, plain_small):
    """fx_attention_tree (one call over the hierarchy) gives the same levels
    and top-k lists as one fx_attention call per level, and as the oracle."""
    c = plain_small.circuit
    d = fx.Design(ctx, c)
    try:
        tree = d.partition(fx.part_cfg())
        whole = d.attention(tree, top_k=10)
        per_level = d.attention(tree, top_k=10, scores=True)
        one = d.attention(tree, top_k=1)
        # malformed trees are refused
        with pytest.raises(fx.FluxionError):
            d.attention(dict(tree, leaf_depth=np.ones_like(tree["leaf_depth"])), top_k=10)
    finally:
        d.close()
    assert [lv["level_index"] for lv in whole] == [lv["level_index"] for lv in per_level]
    assert all(np.array_equal(a["top_k"], b["top_k"]) for a, b in zip(whole, per_level))
    assert all(np.array_equal(a["top_k"], b["top_k"][:, :1]) for a, b in zip(one, whole))
    levels = fx.hierarchy_levels(tree["leaf_ptr"], tree["leaf_gate"], tree["leaf_depth"])
    for lv in whole:
        cp, cg = levels[lv["level_index"]]
        _, _, _, tk = oracle.attention_level_sparse(c.net_ptr, c.net_gate, c.num_gates, cp, cg,
                                                    10)
        assert fx.top_k_lists(lv["top_k"]) == fx.top_k_lists(tk)

"""Attention scoring on the CPU: the oracle against the reference's known
answer, the vectorised oracle against the literal one, and the host-side
level extraction (clusters_at_depth) against the oracle's explicit tree.
"""
import numpy as np
import pytest


def _random_level(rng, n_gates, n_nets, n_clusters, max_pins=6, outside=0.1):
    sizes = rng.integers(2, max_pins + 1, n_nets)
    net_ptr = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int32)
    net_gate = rng.integers(0, n_gates, int(sizes.sum())).astype(np.int32)
    gates = rng.permutation(n_gates)
    gates = gates[: int(n_gates * (1 - outside))]
    cuts = np.sort(rng.choice(np.arange(1, len(gates)), n_clusters - 1, replace=False))
    cluster_ptr = np.concatenate([[0], cuts, [len(gates)]]).astype(np.int32)
    return net_ptr, net_gate, cluster_ptr, gates.astype(np.int32)


def test_attention_basic_known_answer(oracle):
    # HAPR_fluxion_v4/src/algorithm/attention.rs:107-126: clusters {0,1,2} and
    # {3,4,5}; nets {0,1}, {0,3}, {3,4}. Each cluster touches two nets, one shared.
    net_ptr, net_gate = [0, 2, 4, 6], [0, 1, 0, 3, 3, 4]
    s, top = oracle.attention_level(net_ptr, net_gate, [[0, 1, 2], [3, 4, 5]], top_k=5)
    assert s.tolist() == [[0.0, 0.5], [0.5, 0.0]]
    assert top == [[1], [0]]
    # the tree of that test: a root over two leaves at depth 1
    levels = oracle.attention_all(net_ptr, net_gate, [0, 3, 6], [0, 1, 2, 3, 4, 5], [1, 1], 5)
    assert [d for d, _, _ in levels] == [1]


def test_attention_top_k_order_and_zero_drop(oracle):
    # cluster 0 touches four nets: scores 1/4 to clusters 1 and 3 (a tie kept
    # in index order), 2/4 to 2; cluster 4 shares nothing and is dropped even
    # when top_k reaches it
    clusters = [[0], [1], [2], [3], [4]]
    net_ptr, net_gate = [0, 2, 4, 6], [0, 2, 0, 1, 0, 3]
    net_ptr += [8]
    net_gate = net_gate + [2, 0]
    s, top = oracle.attention_level(net_ptr, net_gate, clusters, top_k=10)
    assert s[0].tolist() == [0.0, np.float32(1) / np.float32(4), np.float32(2) / np.float32(4),
                             np.float32(1) / np.float32(4), 0.0]
    assert top[0] == [2, 1, 3]
    _, top2 = oracle.attention_level(net_ptr, net_gate, clusters, top_k=2)
    assert top2[0] == [2, 1]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_sparse_oracle_matches_literal(oracle, seed):
    rng = np.random.default_rng(seed)
    n_gates, n_clusters = 300, 23
    net_ptr, net_gate, cp, cg = _random_level(rng, n_gates, 260, n_clusters)
    # a net naming one gate twice, and a cluster that touches no net
    net_gate[1] = net_gate[0]
    clusters = [cg[cp[i]:cp[i + 1]].tolist() for i in range(n_clusters)]
    for top_k in (0, 1, 3, 40):
        s, top = oracle.attention_level(net_ptr, net_gate, clusters, top_k)
        r, c, v, tk = oracle.attention_level_sparse(net_ptr, net_gate, n_gates, cp, cg, top_k)
        dense = np.zeros_like(s)
        dense[r, c] = v
        assert np.array_equal(dense.view(np.uint32), s.view(np.uint32))
        assert [[j for j in row if j >= 0] for row in tk.tolist()] == top


def _hand_tree():
    # root -> (A, B); A -> (a0, a1); B leaf; a1 -> (x, y): leaves a0, x, y, B
    leaf_depth = [2, 3, 3, 1]
    leaf_ptr = [0, 2, 3, 5, 9]
    leaf_gate = [4, 0, 8, 1, 2, 3, 5, 6, 7]
    return leaf_ptr, leaf_gate, leaf_depth


def test_hierarchy_levels_hand_tree(fx, oracle):
    lp, lg, ld = _hand_tree()
    levels = fx.hierarchy_levels(lp, lg, ld)
    nodes = oracle.hierarchy_nodes(lp, lg, ld)
    assert len(levels) == 4
    for depth, (cp, cg) in enumerate(levels):
        want = oracle.clusters_at_depth(nodes, depth)
        got = [cg[cp[i]:cp[i + 1]].tolist() for i in range(len(cp) - 1)]
        assert got == want
    cp, cg = levels[1]
    assert [cg[cp[i]:cp[i + 1]].tolist() for i in range(2)] == [[4, 0, 8, 1, 2], [3, 5, 6, 7]]


def test_hierarchy_levels_rejects_non_binary_depths(fx):
    with pytest.raises(ValueError):
        fx.hierarchy_levels([0, 1, 2, 3], [0, 1, 2], [1, 1, 1])
    with pytest.raises(ValueError):
        fx.hierarchy_levels([0, 1, 2], [0, 1], [1, 2])


def test_hierarchy_levels_on_the_oracle_hierarchy(fx, oracle):
    s = fx.synth_plain(7, 3000, 3600, 64.0)
    c = s.circuit
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    t = oracle.build_hierarchy(c.num_gates, ap, ai, c.chip_width, c.chip_height)
    levels = fx.hierarchy_levels(t["leaf_ptr"], t["leaf_gate"], t["leaf_depth"])
    nodes = oracle.hierarchy_nodes(t["leaf_ptr"], t["leaf_gate"], t["leaf_depth"])
    assert len(levels) == t["max_depth"] + 1
    assert len(nodes) == t["num_nodes"]
    for depth, (cp, cg) in enumerate(levels):
        want = oracle.clusters_at_depth(nodes, depth)
        assert len(cp) - 1 == len(want)
        assert all(cg[cp[i]:cp[i + 1]].tolist() == list(want[i]) for i in range(len(want)))


@pytest.mark.parametrize("top_k", [0, 2, 10])
def test_cpp_oracle_matches_python(oracle, top_k):
    rng = np.random.default_rng(5)
    net_ptr, net_gate, cp, cg = _random_level(rng, 250, 220, 19)
    net_gate[3] = net_gate[2]
    clusters = [cg[cp[i]:cp[i + 1]].tolist() for i in range(19)]
    s, top = oracle.attention_level(net_ptr, net_gate, clusters, top_k)
    sc, tk, t = oracle.attention_sample(net_ptr, net_gate, cp, cg, np.arange(19), top_k)
    assert np.array_equal(sc.view(np.uint32), s.view(np.uint32))
    assert [[j for j in r if j >= 0] for r in tk.tolist()] == top
    assert np.all(t >= 0)
    # a sample of rows sees the same scores among the sampled clusters
    rows = np.array([3, 7, 11, 18])
    sc2, _, _ = oracle.attention_sample(net_ptr, net_gate, cp, cg, rows, top_k)
    assert np.array_equal(sc2, s[np.ix_(rows, rows)])

"""fx_partition (build_hierarchy, partitioner.rs:36-100, + the leaf regions of
placer.rs:40-63) against the oracle's restatement of the reference."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _oracle_tree(oracle, fx, c, cfg):
    ap, ai = fx.build_adjacency(c)
    return oracle.build_hierarchy(c.num_gates, ap, ai, c.chip_width, c.chip_height,
                                  cfg.max_leaf_size, cfg.min_cluster_size, cfg.balance_factor,
                                  cfg.power_iterations)


def _same_tree(got, ref):
    assert np.array_equal(got["leaf_ptr"], ref["leaf_ptr"])
    assert np.array_equal(got["leaf_gate"], ref["leaf_gate"])
    assert np.array_equal(got["region"], ref["region"])
    assert np.array_equal(got["leaf_depth"], ref["leaf_depth"])
    assert got["num_nodes"] == ref["num_nodes"] and got["max_depth"] == ref["max_depth"]


def _cut(c, leaf_ptr, leaf_gate):
    """Nets whose gates span more than one leaf."""
    leaf_of = np.empty(c.num_gates, np.int64)
    for l in range(len(leaf_ptr) - 1):
        leaf_of[leaf_gate[leaf_ptr[l]:leaf_ptr[l + 1]]] = l
    cut = 0
    for e in range(c.num_nets):
        g = c.net_gate[c.net_ptr[e]:c.net_ptr[e + 1]]
        cut += len(g) > 1 and len(np.unique(leaf_of[g])) > 1
    return cut


def test_partition_chain_matches_reference_test(fx, ctx, oracle):
    """partitioner.rs:232-251: a 20-gate chain with max_leaf_size 8 covers every gate."""
    c = fx.Circuit.from_nets([[i, i + 1] for i in range(19)], 20)
    cfg = fx.part_cfg(max_leaf_size=8)
    d = fx.Design(ctx, c)
    try:
        got = d.partition(cfg)
    finally:
        d.close()
    assert got["max_depth"] >= 1 and len(got["leaf_ptr"]) - 1 >= 2
    assert np.array_equal(np.sort(got["leaf_gate"]), np.arange(20))
    _same_tree(got, _oracle_tree(oracle, fx, c, cfg))


@pytest.mark.parametrize("n,m,die", [(10_000, 12_000, 120.0), (50_000, 60_000, 268.0)])
def test_partition_exact_is_identical_to_the_reference(fx, ctx, oracle, n, m, die):
    s = fx.synth_plain(42, n, m, die)
    cfg = fx.part_cfg()
    d = fx.Design(ctx, s.circuit)
    try:
        got = d.partition(cfg)
    finally:
        d.close()
    ref = _oracle_tree(oracle, fx, s.circuit, cfg)
    _same_tree(got, ref)
    assert got["power_iterations"] > 0


def test_partition_small_designs(fx, ctx, oracle):
    for n in (1, 8, 64, 65, 130):
        c = fx.Circuit.from_nets([[i, (i + 1) % n] for i in range(n - 1)] if n > 1 else [], n)
        cfg = fx.part_cfg()
        d = fx.Design(ctx, c)
        try:
            got = d.partition(cfg)
        finally:
            d.close()
        _same_tree(got, _oracle_tree(oracle, fx, c, cfg))


def test_partition_fp64_mode_same_shape_and_cut(fx, ctx):
    """FX_PART_FP64 (FP64 norms, Rayleigh-quotient stop at tol, up to 500
    iterations): the tree shape depends only on sizes, so leaf sizes,
    regions and depths equal the exact mode's; the leaves cover every gate
    once and cut no more nets than the reference's 30-iteration bisection
    (+10 %)."""
    s = fx.synth_plain(7, 20_000, 24_000, 170.0)
    d = fx.Design(ctx, s.circuit)
    try:
        ex = d.partition(fx.part_cfg())
        fp = d.partition(fx.part_cfg(mode=fx.FX_PART_FP64, power_iterations=500, tol=1e-6))
    finally:
        d.close()
    assert np.array_equal(fp["leaf_ptr"], ex["leaf_ptr"])
    assert np.array_equal(fp["region"], ex["region"])
    assert np.array_equal(fp["leaf_depth"], ex["leaf_depth"])
    assert np.array_equal(np.sort(fp["leaf_gate"]), np.arange(20_000))
    assert _cut(s.circuit, fp["leaf_ptr"], fp["leaf_gate"]) <= \
        1.10 * _cut(s.circuit, ex["leaf_ptr"], ex["leaf_gate"])


def test_partition_rejects_bad_config_and_small_capacity(fx, ctx, plain_small):
    d = fx.Design(ctx, plain_small.circuit)
    try:
        with pytest.raises(fx.FluxionError):
            d.partition(fx.part_cfg(balance_factor=0.7))
        with pytest.raises(fx.FluxionError):
            d.partition(fx.part_cfg(mode=5))
        import ctypes as C
        lp = np.zeros(3, np.int32)
        rc = d.lib.fx_partition(ctx.handle, d.handle, C.byref(fx.part_cfg()), 2,
                                lp.ctypes.data_as(C.POINTER(C.c_int32)), None, None, None, None)
        assert rc == -1
    finally:
        d.close()

"""Barnes-Hut deep keys in the oracle (CPU): when a level-15 cell of the root
square is not accepted by every point, the tree continues 12 levels below
it, so crowded cells are opened level by level instead of point by point."""
import numpy as np

F32_01 = float(np.float32(0.1))


def _crowded(die, seed=3, clusters=3, per=1500, spread=0.005, background=2000):
    rng = np.random.default_rng(seed)
    pts = [rng.uniform(0, die, (background, 2))]
    for _ in range(clusters):
        ctr = rng.uniform(100, die - 100, 2)
        pts.append(ctr + rng.uniform(0, spread, (per, 2)))
    p = np.concatenate(pts).astype(np.float32)
    return p[:, 0].copy(), p[:, 1].copy()


def test_deep_tree_on_a_large_die_is_accurate_and_shallow_per_point(oracle):
    # die 4000: a level-15 cell (~0.122) exceeds theta * min_dist = 0.05
    x, y = _crowded(4000.0)
    o = oracle.bh_forces(x, y, 0.5, 0.5, F32_01)
    ex, ey = oracle.repulsion_exact(x, y, 0.5, F32_01)
    num = np.sqrt(((o["fx"] - ex) ** 2 + (o["fy"] - ey) ** 2).sum())
    den = np.sqrt((ex ** 2 + ey ** 2).sum())
    assert num / den < 1e-5
    # a clustered point no longer interacts with its 1500 neighbours one by one
    assert o["interactions"].max() < 400


def test_small_die_keeps_the_30_bit_tree(oracle):
    # die 1000: level-15 cells (~0.031) are accepted whole; the points of one
    # cell stay one bucket, and the clustered points see few interactions
    x, y = _crowded(1000.0, seed=4)
    o = oracle.bh_forces(x, y, 0.5, 0.5, F32_01)
    assert o["interactions"].max() < 400
    ex, ey = oracle.repulsion_exact(x, y, 0.5, F32_01)
    num = np.sqrt(((o["fx"] - ex) ** 2 + (o["fy"] - ey) ** 2).sum())
    assert num / np.sqrt((ex ** 2 + ey ** 2).sum()) < 1e-5

"""The CPU oracle against fixtures produced by the reference itself.

Fixtures come from tests/golden/make_golden.py, which runs the reference's own
force_electrostatic.py and its own BarnesHutTree.cpp.
"""
import numpy as np
import pytest


@pytest.mark.parametrize("G", [64, 128])
def test_poisson_solve_matches_reference(oracle, golden, G):
    d = golden["dct"]
    wx, wy = d[f"solve{G}_w"]
    phi, ex, ey = oracle.solve_poisson(d[f"solve{G}_rho"], wx, wy)
    for a, b in ((phi, d[f"solve{G}_phi"]), (ex, d[f"solve{G}_ex"]), (ey, d[f"solve{G}_ey"])):
        assert np.allclose(a, b, rtol=1e-12, atol=1e-12 * np.abs(b).max())


def test_density_forces_match_reference(oracle, golden):
    d = golden["dct"]
    G, die, target, weight = d["calc_meta"]
    out = oracle.density_forces(d["calc_x"], d["calc_y"], d["calc_area"], die, die,
                                int(G), target, weight)
    ref = d["calc_forces"]
    assert np.allclose(out["fx"], ref[:, 0], rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    assert np.allclose(out["fy"], ref[:, 1], rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    assert abs(out["energy"] - d["calc_energy"][0]) <= 1e-9 * abs(d["calc_energy"][0])


def _rel(ax, ay, bx, by):
    return np.sqrt(((ax - bx) ** 2 + (ay - by) ** 2).sum() / (bx ** 2 + by ** 2).sum())


@pytest.mark.parametrize("name", ["uniform", "clustered", "small"])
def test_force_law_matches_reference_tree_at_theta0(oracle, golden, name):
    # theta = 0 opens every node: the reference tree then sums all pairs with
    # its law k q Q / max(d, min_dist)^2; the oracle's exact sum must agree.
    b = golden["bh"]
    x, y = b[f"bh_{name}_x"], b[f"bh_{name}_y"]
    fx, fy = oracle.repulsion_exact(x, y, 0.5, 0.1)
    assert _rel(fx, fy, b[f"bh_{name}_t0_fx"], b[f"bh_{name}_t0_fy"]) < 1e-12
    o = oracle.bh_forces(x, y, 0.5, 0.0, 0.1)
    assert _rel(o["fx"], o["fy"], b[f"bh_{name}_t0_fx"], b[f"bh_{name}_t0_fy"]) < 1e-12


@pytest.mark.parametrize("name", ["uniform", "clustered", "small"])
def test_barnes_hut_matches_reference_tree(oracle, golden, name):
    # theta = 0.5: same opening rule and quadrant convention as the reference
    # tree; the trees differ only in precision (f32 vs f64 decisions) and
    # below 15 levels, so most points see the same interaction list.
    b = golden["bh"]
    x, y = b[f"bh_{name}_x"], b[f"bh_{name}_y"]
    rx, ry = b[f"bh_{name}_t05_fx"], b[f"bh_{name}_t05_fy"]
    o = oracle.bh_forces(x, y, 0.5, 0.5, 0.1)
    per = np.hypot(o["fx"] - rx, o["fy"] - ry) / np.maximum(np.hypot(rx, ry), 1e-30)
    assert np.median(per) < 1e-9
    assert np.mean(per < 1e-6) > 0.95
    assert _rel(o["fx"], o["fy"], rx, ry) < 2e-3
    ex_x, ex_y = oracle.repulsion_exact(x, y, 0.5, 0.1)
    assert _rel(o["fx"], o["fy"], ex_x, ex_y) < 2e-2


def test_morton_keys_boundary_rule(oracle):
    # A point exactly on a cell's midline belongs to the lower (west/south)
    # half, as `px <= mx` in BarnesHutTree.cpp:107-123.
    root = np.array([0.0, 0.0, 32768.0], np.float32)
    k = oracle.bh_keys(np.array([16384.0, 16384.5, 0.0], np.float32),
                       np.array([0.0, 0.0, 32768.0], np.float32), root)
    assert (k[0] >> 29) & 1 == 0 and (k[1] >> 29) & 1 == 1
    assert k[2] == 0x15555555  # x cell 0, y cell 32767

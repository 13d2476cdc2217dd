"""Row G: batched power iteration against compute_fiedler_vector
(HAPR_fluxion_v4/src/algorithm/partitioner.rs:106-185), restated in the
oracle with the reference's f32 arithmetic."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _laplacian(ap, ai, g, x):
    """L x of the cluster's induced Laplacian (partitioner.rs:124-137), FP64."""
    pos = {int(q): i for i, q in enumerate(g)}
    x = np.asarray(x, np.float64)
    lx = np.zeros_like(x)
    for i, q in enumerate(g):
        nb = [pos[int(j)] for j in ai[ap[q]:ap[q + 1]] if int(j) in pos]
        lx[i] = len(nb) * x[i] - x[nb].sum()
    return lx


def _rayleigh(ap, ai, g, v):
    x = np.asarray(v, np.float64)
    return float(x @ _laplacian(ap, ai, g, x)) / float(x @ x)


def test_power_iteration_matches_reference(fx, ctx, oracle):
    s = fx.synth_plain(21, 6000, 7200, 85.0)
    c = s.circuit
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    # the two clusters of the first bisection level plus the root's halves
    rng = np.random.default_rng(2)
    perm = rng.permutation(c.num_gates).astype(np.int32)
    cp = np.array([0, 1500, 1564, 4000, 6000], np.int32)  # incl. a 64-gate cluster
    d = fx.Design(ctx, c)
    try:
        v, its, lam = d.fiedler(cp, perm, max_iters=30)
    finally:
        d.close()
    assert np.all(its == 30)
    for k in range(len(cp) - 1):
        ref = oracle.fiedler_vector(ap, ai, perm[cp[k]:cp[k + 1]], iters=30)
        got = v[cp[k]:cp[k + 1]]
        assert np.array_equal(got, ref), k  # the reference's f32 folds: bit-identical
        assert abs(np.linalg.norm(got.astype(np.float64)) - 1.0) < 1e-5
        assert abs(_rayleigh(ap, ai, perm[cp[k]:cp[k + 1]], got) - lam[k]) <= 1e-6 * lam[k]


def test_power_iteration_tolerance_mode(fx, ctx, oracle):
    """tol > 0: every cluster stops by its Rayleigh-quotient criterion within
    the iteration cap, and the quotient matches a float64 recomputation."""
    s = fx.synth_plain(22, 4000, 4800, 70.0)
    c = s.circuit
    ap, ai = oracle.build_adjacency(c.num_gates, c.net_ptr, c.net_gate)
    cp = np.array([0, 2000, 4000], np.int32)
    gates = np.arange(4000, dtype=np.int32)
    d = fx.Design(ctx, c)
    try:
        v, its, lam = d.fiedler(cp, gates, max_iters=500, tol=1e-6)
    finally:
        d.close()
    assert np.all(its <= 500) and np.all(its > 1)
    for k in range(2):
        rq = _rayleigh(ap, ai, gates[cp[k]:cp[k + 1]], v[cp[k]:cp[k + 1]])
        assert abs(rq - lam[k]) <= 1e-6 * abs(rq)
        # converged: one more iteration (FP64) moves the quotient by ~tol at most
        x = v[cp[k]:cp[k + 1]].astype(np.float64)
        y = _laplacian(ap, ai, gates[cp[k]:cp[k + 1]], x)
        y -= y.mean()
        y /= np.linalg.norm(y)
        assert abs(_rayleigh(ap, ai, gates[cp[k]:cp[k + 1]], y) - rq) <= 1e-5 * abs(rq)


def test_singletons_and_empty_clusters(fx, ctx):
    s = fx.synth_plain(23, 300, 360, 20.0)
    d = fx.Design(ctx, s.circuit)
    try:
        cp = np.array([0, 1, 1, 300], np.int32)
        v, its, _ = d.fiedler(cp, np.arange(300, dtype=np.int32), max_iters=5)
    finally:
        d.close()
    assert v[0] == 0.0 and np.all(np.isfinite(v))

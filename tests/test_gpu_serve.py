"""The request server (fx_serve_*): every job gives the same result in a mix
of concurrent jobs as alone, admission follows the device budget, and jobs
on one design run in submission order."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _designs(fx):
    sizes = [(5_000, 6_000), (12_000, 14_400), (8_000, 9_600), (20_000, 24_000)]
    return [fx.synth_plain(100 + i, n, m, 1.2 * float(np.sqrt(n))).circuit
            for i, (n, m) in enumerate(sizes)]


def _moves(c, seed, frac=0.01, sigma=None):
    rng = np.random.default_rng(seed)
    k = max(1, int(frac * c.num_gates))
    g = rng.choice(c.num_gates, k, replace=False).astype(np.int32)
    sig = sigma if sigma is not None else 2.0 * c.chip_width / 128
    return g, rng.normal(0, sig, k).astype(np.float32), rng.normal(0, sig, k).astype(np.float32)


def _key(r):
    return (r["status"], r["hpwl"], r["total_overflow"], r["max_overflow"], r["iterations"],
            r["n_leaves"])


def _run(fx, circuits, slots, alone):
    """PLACE every circuit (the first two stay resident), then two ECO jobs on
    each resident design. alone: one job at a time, waiting for each."""
    sv = fx.Server(slots=slots)
    try:
        res, order = {}, []

        def go(desc):
            jid = sv.submit(desc)
            order.append(jid)
            if alone:
                r = sv.poll(-1)
                res[r["job_id"]] = r
            return jid

        ids = [go(sv.place_desc(c, keep_resident=i < 2)) for i, c in enumerate(circuits)]
        for rnd in range(2):
            for i in range(2):
                g, dx, dy = _moves(circuits[i], 10 * rnd + i)
                go(sv.eco_desc(ids[i], g, dx, dy, iterations=20))
        while len(res) < len(order):
            r = sv.poll(-1)
            assert r is not None
            res[r["job_id"]] = r
        pos = [sv.positions(ids[i], circuits[i].num_gates) for i in range(2)]
    finally:
        sv.close()
    return [res[j] for j in order], pos


def test_results_are_the_same_alone_and_in_the_mix(fx):
    circuits = _designs(fx)
    mix, pos_mix = _run(fx, circuits, slots=6, alone=False)
    solo, pos_solo = _run(fx, circuits, slots=1, alone=True)
    for a, b in zip(mix, solo):
        assert a["status"] == 0, a["error"]
        assert _key(a) == _key(b)  # bit-identical statistics
    for (xa, ya), (xb, yb) in zip(pos_mix, pos_solo):
        assert np.array_equal(xa, xb) and np.array_equal(ya, yb)
    # the mix really overlapped: some job started before another ended
    spans = sorted((r["start_s"], r["end_s"]) for r in mix)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))


def test_place_job_matches_the_direct_calls(fx, ctx):
    """A PLACE job is fx_partition -> fx_hapr_place_leaves (tolerance-mode
    forces, the server's default) -> fx_refine."""
    c = _designs(fx)[0]
    sv = fx.Server(slots=2)
    try:
        jid = sv.submit_place(c, keep_resident=True)
        r = sv.poll(-1)
        x, y = sv.positions(jid, c.num_gates)
    finally:
        sv.close()
    d = fx.Design(ctx, c)
    try:
        t = d.partition()
        lx, ly, _ = d.place_leaves(t["leaf_ptr"], t["leaf_gate"], t["region"].reshape(-1),
                                   fx.leaf_cfg(precision=fx.FX_LEAF_FAST))
        st = d.refine(fx.refine_cfg(), lx, ly)
    finally:
        d.close()
    assert r["status"] == 0 and r["n_leaves"] == len(t["leaf_ptr"]) - 1
    assert r["hpwl"] == st.hpwl and r["iterations"] == st.iterations
    assert np.array_equal(x, lx) and np.array_equal(y, ly)


def test_admission_by_budget(fx):
    c = _designs(fx)[0]
    desc = fx.Server.place_desc(c)
    est = fx.serve_estimate(desc)
    small = fx.Server(slots=4, hbm_budget_bytes=est // 2)
    try:
        with pytest.raises(fx.FluxionError) as e:
            small.submit(desc)
        assert e.value.code == -5  # FX_EADMIT
    finally:
        small.close()
    # room for one job at a time: the second starts after the first ends
    one = fx.Server(slots=4, hbm_budget_bytes=int(est * 1.5))
    try:
        a = one.submit(fx.Server.place_desc(c))
        b = one.submit(fx.Server.place_desc(c))
        rs = {r["job_id"]: r for r in (one.poll(-1), one.poll(-1))}
        assert rs[b]["start_s"] >= rs[a]["end_s"] and rs[a]["hpwl"] == rs[b]["hpwl"]
        assert one.stats()["reserved_bytes"] == 0
    finally:
        one.close()


def test_eco_on_unknown_or_released_design(fx):
    c = _designs(fx)[0]
    sv = fx.Server(slots=2)
    try:
        g, dx, dy = _moves(c, 1)
        with pytest.raises(fx.FluxionError):
            sv.submit_eco(12345, g, dx, dy)
        jid = sv.submit_place(c, keep_resident=True)
        assert sv.poll(-1)["status"] == 0
        assert sv.stats()["resident"] == 1
        sv.release(jid)
        st = sv.stats()
        assert (st["reserved_bytes"], st["queued"], st["running"], st["resident"]) == (0, 0, 0, 0)
        assert st["launches"] > 0
        with pytest.raises(fx.FluxionError):
            sv.submit_eco(jid, g, dx, dy)
        bad = sv.submit_place(c, keep_resident=True)
        assert sv.poll(-1)["status"] == 0
        sv.submit_eco(bad, np.array([c.num_gates + 5], np.int32), np.zeros(1), np.zeros(1))
        r = sv.poll(-1)
        assert r["status"] == -1 and "outside" in r["error"]
        sv.submit_eco(bad, np.array([3, 9, 3], np.int32), np.ones(3), np.ones(3))
        r = sv.poll(-1)
        assert r["status"] == -1 and "twice" in r["error"]
    finally:
        sv.close()

"""Single-iteration calls of fx_force_iterate on resident positions replay a
cached CUDA graph of the call after two eager calls of the same parity and
configuration. Replayed calls must give the eager calls' results bit for
bit, and a changed configuration must not replay a stale graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run(fx, ctx, d, cfg, calls, eager):
    """`calls` single-iteration calls, each from the saved state; eager=True
    turns the force trace on, under which every call runs without a graph."""
    d.trace(eager)
    out = []
    try:
        for _ in range(calls):
            d.restore_state()
            l0 = ctx.kernel_launches()
            st = d.force_iterate(cfg, 1)
            x, y = d.get_positions()
            out.append((x, y, st.hpwl, st.total_overflow, st.max_overflow,
                        st.density_energy, ctx.kernel_launches() - l0))
    finally:
        d.trace(False)
    return out


def _same(a, b):
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert a[2:] == b[2:]


@pytest.mark.parametrize("walk", ["fast", "exact"])
def test_replayed_single_steps_match_eager(fx, ctx, walk):
    s = fx.synth_plain(31, 20000, 24000, 170.0)
    d = fx.Design(ctx, s.circuit)
    try:
        cfg = fx.iter_cfg(density_bins=128, cong_cols=64, cong_rows=64,
                          bh_walk=fx.FX_BH_FAST if walk == "fast" else fx.FX_BH_EXACT)
        d.set_positions(s.placement.gate_x, s.placement.gate_y)
        d.save_state()
        ref = _run(fx, ctx, d, cfg, 2, eager=True)  # one call per parity
        # eager, eager, captured, captured, then replays; parities alternate
        got = _run(fx, ctx, d, cfg, 8, eager=False)
        for i, g in enumerate(got):
            _same(g, ref[i % 2])
        # a different configuration on the same design: no stale replay
        cfg2 = fx.iter_cfg(density_bins=128, cong_cols=64, cong_rows=64, density_weight=2e-4,
                           bh_walk=cfg.bh_walk)
        ref2 = _run(fx, ctx, d, cfg2, 2, eager=True)
        got2 = _run(fx, ctx, d, cfg2, 6, eager=False)
        for i, g in enumerate(got2):
            _same(g, ref2[i % 2])
        # and back: the first configuration's results again
        got3 = _run(fx, ctx, d, cfg, 4, eager=False)
        for i, g in enumerate(got3):
            _same(g, ref[i % 2])
    finally:
        d.close()


def test_replay_after_positions_change(fx, ctx):
    """New positions through fx_design_set_positions between calls: every
    call's result is that of an eager call from the same positions."""
    s = fx.synth_plain(32, 12000, 14400, 130.0)
    d = fx.Design(ctx, s.circuit)
    try:
        cfg = fx.iter_cfg(density_bins=128, cong_cols=64, cong_rows=64)
        rng = np.random.default_rng(5)
        states = [(rng.uniform(0, 130.0, s.circuit.num_gates).astype(np.float32),
                   rng.uniform(0, 130.0, s.circuit.num_gates).astype(np.float32))
                  for _ in range(3)]
        def one(x, y, eager):
            d.trace(eager)
            try:
                d.set_positions(x, y)
                st = d.force_iterate(cfg, 1)
                return d.get_positions(), (st.hpwl, st.total_overflow, st.max_overflow)
            finally:
                d.trace(False)
        for k in range(12):
            x, y = states[k % 3]
            (gx, gy), gs = one(x, y, eager=False)
            (rx, ry), rs = one(x, y, eager=True)
            assert np.array_equal(gx, rx) and np.array_equal(gy, ry) and gs == rs, k
    finally:
        d.close()


def test_stage_times_count_every_call(fx, ctx):
    """With stage timing on, single-iteration calls still replay a cached
    graph, which records the timed stages' events itself: each call adds the
    walk's and the density solve's times once, and the results stay those of
    eager calls."""
    s = fx.synth_plain(33, 20000, 24000, 170.0)
    d = fx.Design(ctx, s.circuit)
    try:
        cfg = fx.iter_cfg(density_bins=128, cong_cols=64, cong_rows=64)
        d.set_positions(s.placement.gate_x, s.placement.gate_y)
        d.save_state()
        ref = _run(fx, ctx, d, cfg, 2, eager=True)
        ctx.reset_stage_times()
        ctx.set_profiling(True, stages=("bh_walk", "density"))
        try:
            got = _run(fx, ctx, d, cfg, 10, eager=False)
        finally:
            ctx.set_profiling(False)
        for i, g in enumerate(got):
            _same(g, ref[i % 2])
        t = ctx.stage_times()
        assert t["bh_walk"][1] == 10 and t["density"][1] == 10
        assert t["bh_walk"][0] > 0 and t["density"][0] > 0
        assert t["bh_sort"][1] == 0  # not in the mask
        # the replays' walk times are of the same order as the eager calls'
        ctx.reset_stage_times()
        ctx.set_profiling(True, stages=("bh_walk",))
        try:
            _run(fx, ctx, d, cfg, 2, eager=True)
        finally:
            ctx.set_profiling(False)
        te = ctx.stage_times()["bh_walk"]
        assert te[1] == 2
        assert 0.2 < (t["bh_walk"][0] / 10) / (te[0] / 2) < 5.0
    finally:
        d.close()
